/*
 * Test infrastructure only: a plain-C restatement of the reference
 * simulator's CPU double-precision arithmetic (Line-fr/Kate). It is the
 * checker for the CUDA path; nothing in the product links or loads it.
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own CPU path, compiled from its headers into oracle/_ref/
 * (oracle/ref_harness.cpp), and against the committed fixtures in
 * tests/golden/.
 *
 * State layout: 2^n interleaved (re, im) doubles; qubit q is bit q of the
 * amplitude index (little-endian), as in the reference.
 *
 * The arithmetic follows the reference operation by operation, so that a
 * build with the same flags (no FP contraction) is bit-identical to it:
 *   gate kernels     CPUcode/GateComputing.hpp:6-129
 *   Complex ops      backendagnosticcode/basic_host_types.hpp:34-78
 *   gate merging     CPUcode/GateMerger.hpp:8-55
 *   initialisation   CPUcode/simulator.hpp:133-162
 *   measurement      CPUcode/simulator.hpp:163-197
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KO_PI 3.1415926535897932384626433
#define KO_SQRT2 1.4142135623730951
#define KO_SQRT2INV 0.7071067811865475

typedef struct { double a, b; } ko_c;

static inline ko_c c_add(ko_c x, ko_c y) { ko_c r = {x.a + y.a, x.b + y.b}; return r; }
static inline ko_c c_sub(ko_c x, ko_c y) { ko_c r = {x.a - y.a, x.b - y.b}; return r; }
/* operator*(Complex): (a*c - b*d, a*d + b*c)  basic_host_types.hpp:43-45 */
static inline ko_c c_mul(ko_c x, ko_c y) { ko_c r = {x.a * y.a - x.b * y.b, x.a * y.b + x.b * y.a}; return r; }
static inline ko_c c_muld(ko_c x, double d) { ko_c r = {x.a * d, x.b * d}; return r; }
/* operator*=(Complex): a' = a*c - b*d; b' = a*d + b*c  basic_host_types.hpp:69-73 */
static inline ko_c c_mul_assign(ko_c x, ko_c y) {
    double t = x.a;
    ko_c r;
    r.a = x.a * y.a - x.b * y.b;
    r.b = t * y.b + x.b * y.a;
    return r;
}
/* operator/(Complex)  basic_host_types.hpp:54-57 */
static inline ko_c c_div(ko_c x, ko_c y) {
    double n = y.a * y.a + y.b * y.b;
    ko_c r = {(x.a * y.a + x.b * y.b) / n, (y.a * x.b - x.a * y.b) / n};
    return r;
}
static inline double c_norm(ko_c x) { return sqrt(x.a * x.a + x.b * x.b); }
static inline double c_angle(ko_c x) { return atan(x.b / x.a); }

/* Inserts zero bits at the (ascending) positions pos[0..k-1] of `line`. */
static uint64_t insert_zeros(uint64_t line, const int* sorted_pos, int k) {
    uint64_t v = line;
    for (int i = 0; i < k; i++) {
        uint64_t p = (uint64_t)sorted_pos[i];
        uint64_t low = v & ((1ull << p) - 1);
        v = ((v >> p) << (p + 1)) | low;
    }
    return v;
}

static void sort_ints(int* v, int k) {
    for (int i = 1; i < k; i++) {
        int x = v[i], j = i - 1;
        while (j >= 0 && v[j] > x) { v[j + 1] = v[j]; j--; }
        v[j + 1] = x;
    }
}

/*
 * Applies one gate to the 2^n state `st` (ko_c array). Qubit indices are
 * state bit positions. ids: 0 dense (row-major 2^k x 2^k, bit i of the
 * gate-local index <-> qbits[i]), 2 H, 3 CNOT (qbits[0] target, qbits[1]
 * control), 4 CRk (phase e^{2 pi i / 2^optarg} on |11>), 5 TOFFOLI
 * (qbits[0..1] controls, qbits[2] target). Any other id is a no-op, as in
 * the reference (RX=6 and RZ=7 have no case in computeGate).
 */
static void apply_gate(int n, ko_c* st, int id, int nq, const int* qbits, int optarg, const ko_c* mat) {
    int sorted[64];
    for (int i = 0; i < nq; i++) sorted[i] = qbits[i];
    sort_ints(sorted, nq);
    switch (id) {
    case 5: { /* GateComputing.hpp:8-28 */
        uint64_t cover = 1ull << (n - 3);
        for (uint64_t line = 0; line < cover; line++) {
            uint64_t i110 = insert_zeros(line, sorted, 3) + (1ull << qbits[0]) + (1ull << qbits[1]);
            uint64_t i111 = i110 + (1ull << qbits[2]);
            ko_c t = st[i110];
            st[i110] = st[i111];
            st[i111] = t;
        }
        break;
    }
    case 4: { /* GateComputing.hpp:29-45 */
        uint64_t cover = 1ull << (n - 2);
        for (uint64_t line = 0; line < cover; line++) {
            uint64_t i10 = insert_zeros(line, sorted, 2) + (1ull << qbits[1]);
            uint64_t i11 = i10 + (1ull << qbits[0]);
            double t = ((double)2 * KO_PI) / (double)(1ull << optarg);
            ko_c ph = {cos(t), sin(t)};
            st[i11] = c_mul_assign(st[i11], ph);
        }
        break;
    }
    case 3: { /* GateComputing.hpp:46-64 */
        uint64_t cover = 1ull << (n - 2);
        for (uint64_t line = 0; line < cover; line++) {
            uint64_t i10 = insert_zeros(line, sorted, 2) + (1ull << qbits[1]);
            uint64_t i11 = i10 + (1ull << qbits[0]);
            ko_c t = st[i10];
            st[i10] = st[i11];
            st[i11] = t;
        }
        break;
    }
    case 2: { /* GateComputing.hpp:65-82 */
        uint64_t cover = 1ull << (n - 1);
        for (uint64_t line = 0; line < cover; line++) {
            uint64_t i0 = insert_zeros(line, sorted, 1);
            uint64_t i1 = i0 + (1ull << qbits[0]);
            st[i0] = c_muld(c_add(st[i0], st[i1]), KO_SQRT2INV);
            st[i1] = c_sub(st[i0], c_muld(st[i1], KO_SQRT2));
        }
        break;
    }
    case 0: { /* GateComputing.hpp:83-127 */
        uint64_t cover = 1ull << (n - nq);
        int dim = 1 << nq;
        ko_c cache[32];
        for (uint64_t line = 0; line < cover; line++) {
            uint64_t base = insert_zeros(line, sorted, nq);
            for (int sub = 0; sub < dim; sub++) {
                uint64_t idx = base;
                for (int i = 0; i < nq; i++) idx += (uint64_t)((sub >> i) & 1) << qbits[i];
                cache[sub] = st[idx];
            }
            for (int r = 0; r < dim; r++) {
                ko_c sum = {0.0, 0.0};
                for (int c = 0; c < dim; c++) sum = c_add(sum, c_mul(mat[r * dim + c], cache[c]));
                uint64_t idx = base;
                for (int i = 0; i < nq; i++) idx += (uint64_t)((r >> i) & 1) << qbits[i];
                st[idx] = sum;
            }
        }
        break;
    }
    default:
        break;
    }
}

/* Number of doubles the dense matrix of a gate with nq qubits occupies. */
static size_t dense_len(int nq) { return 2u * ((size_t)1 << (2 * nq)); }

/*
 * Full-state simulation of a gate list from |0...0> (or from the product
 * state given by proba_in, when non-null). Gates are flat arrays: ids[g],
 * nqs[g], qbits (concatenated), optargs[g], dense (concatenated matrices of
 * the dense gates only, in order). state_out: 2*2^n doubles.
 */
int ko_simulate(int n, int ngates, const int* ids, const int* nqs, const int* qbits, const int* optargs,
                const double* dense, const double* proba_in, const int* initial_permutation, double* state_out) {
    ko_c* st = (ko_c*)state_out;
    uint64_t dim = 1ull << n;
    if (proba_in) {
        /* CPUcode/simulator.hpp:139-162 */
        ko_c* all = (ko_c*)malloc(sizeof(ko_c) * 2 * (size_t)n);
        for (int i = 0; i < n; i++) {
            ko_c v0 = {cos(proba_in[2 * i] * KO_PI / 2), 0.0};
            ko_c e = {cos(proba_in[2 * i + 1]), sin(proba_in[2 * i + 1])};
            ko_c v1 = c_muld(e, sin(proba_in[2 * i] * KO_PI / 2));
            int p = initial_permutation ? initial_permutation[i] : i;
            all[p] = v0;
            all[p + n] = v1;
        }
        for (uint64_t i = 0; i < dim; i++) {
            ko_c t = {1.0, 0.0};
            for (int j = 0; j < n; j++) t = c_mul_assign(t, all[((i >> j) & 1) * (uint64_t)n + j]);
            st[i] = t;
        }
        free(all);
    } else {
        memset(st, 0, sizeof(ko_c) * dim);
        st[0].a = 1.0;
    }
    const int* q = qbits;
    const double* d = dense;
    for (int g = 0; g < ngates; g++) {
        const ko_c* mat = NULL;
        if (ids[g] == 0) {
            mat = (const ko_c*)d;
            d += dense_len(nqs[g]);
        }
        apply_gate(n, st, ids[g], nqs[g], q, optargs[g], mat);
        q += nqs[g];
    }
    return 0;
}

/* Applies a single gate to an existing state (2*2^n doubles, in place). */
int ko_apply(int n, double* state, int id, int nq, const int* qbits, int optarg, const double* dense) {
    apply_gate(n, (ko_c*)state, id, nq, qbits, optarg, (const ko_c*)dense);
    return 0;
}

/*
 * Fuses a gate list into one dense gate on the sorted union of its qubits
 * (CPUcode/GateMerger.hpp:8-55): each basis column is simulated through the
 * gates on the local 2^k space, written as a matrix row, and the matrix is
 * transposed. out_qbits receives k sorted qubits, out_dense 2*4^k doubles.
 * Returns k, or -1 if k > 5.
 */
int ko_merge(int ngates, const int* ids, const int* nqs, const int* qbits, const int* optargs, const double* dense,
             int* out_qbits, double* out_dense) {
    int covered[64];
    int k = 0;
    const int* q = qbits;
    for (int g = 0; g < ngates; g++) {
        for (int i = 0; i < nqs[g]; i++) {
            int x = q[i], seen = 0;
            for (int j = 0; j < k; j++) if (covered[j] == x) seen = 1;
            if (!seen) covered[k++] = x;
        }
        q += nqs[g];
    }
    sort_ints(covered, k);
    if (k > 5) return -1;
    int dim = 1 << k;
    ko_c* m = (ko_c*)out_dense;
    for (int r = 0; r < dim; r++)
        for (int c = 0; c < dim; c++) { m[r * dim + c].a = (double)(int)(r == c); m[r * dim + c].b = 0.0; }
    int local[64];
    for (int col = 0; col < dim; col++) {
        q = qbits;
        const double* d = dense;
        for (int g = 0; g < ngates; g++) {
            for (int i = 0; i < nqs[g]; i++) {
                for (int j = 0; j < k; j++) if (covered[j] == q[i]) local[i] = j;
            }
            const ko_c* mat = NULL;
            if (ids[g] == 0) { mat = (const ko_c*)d; d += dense_len(nqs[g]); }
            apply_gate(k, m + (size_t)col * dim, ids[g], nqs[g], local, optargs[g], mat);
            q += nqs[g];
        }
    }
    for (int r = 0; r < dim; r++)
        for (int c = r + 1; c < dim; c++) { ko_c t = m[r * dim + c]; m[r * dim + c] = m[c * dim + r]; m[c * dim + r] = t; }
    for (int i = 0; i < k; i++) out_qbits[i] = covered[i];
    return k;
}

/*
 * The reference's per-qubit measurement (CPUcode/simulator.hpp:163-197):
 * S_b(q) = sum of amplitudes whose bit q is b, scaled by 1/sqrt(2)^n;
 * theta = atan(|S1|/|S0|)/(pi/2), phi = atan(Im/Re of S1/S0), with the
 * reference's thresholds. out[2*final_inv[q]] = theta, [..+1] = phi.
 */
int ko_measure(int n, const double* state, const int* final_inverse_permutation, double* out) {
    const ko_c* st = (const ko_c*)state;
    ko_c* meas = (ko_c*)calloc(2 * (size_t)n, sizeof(ko_c));
    uint64_t dim = 1ull << n;
    for (uint64_t i = 0; i < dim; i++)
        for (int q = 0; q < n; q++) meas[q * 2 + ((i >> q) & 1)] = c_add(meas[q * 2 + ((i >> q) & 1)], st[i]);
    for (int i = 0; i < n; i++) {
        ko_c p = {pow(KO_SQRT2, (double)n), 0.0};
        ko_c v0 = c_div(meas[2 * i], p);
        ko_c v1 = c_div(meas[2 * i + 1], p);
        double teta, phi;
        if (c_norm(v0) < 0.0000000000001) { teta = 1; phi = 0; }
        else if (c_norm(v1) < 0.00000000000001) { teta = 0; phi = 0; }
        else { teta = atan(c_norm(v1) / c_norm(v0)) / (KO_PI / 2); phi = c_angle(c_div(v1, v0)); }
        int o = final_inverse_permutation ? final_inverse_permutation[i] : i;
        out[2 * o] = teta;
        out[2 * o + 1] = phi;
    }
    free(meas);
    return 0;
}
