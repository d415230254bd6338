// Test infrastructure only: a C-ABI harness around the reference simulator's
// own CPU path (Line-fr/Kate, header-only C++). It is compiled from the
// reference headers where they lie (see oracle/Makefile) into oracle/_ref/,
// never copied. Nothing in the product links or loads this library; only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
//
// Reference entry points wrapped here (paths within the reference project):
//   Circuit(int) / appendGate          backendagnosticcode/QuantumCircuit.hpp:18-37
//   Gate(id, qbits, optarg)            backendagnosticcode/basic_host_types.hpp:198-228
//   Gate(Matrix<Complex>, qbits)       backendagnosticcode/basic_host_types.hpp:229-245
//   gateScheduling/gateFusion/gateGrouping/allocate
//                                      backendagnosticcode/Circuit.hpp:12-348
//   compileDefault                     backendagnosticcode/QuantumCircuit.hpp:126-204
//   CPUmergeGate                       CPUcode/GateMerger.hpp:8-55
//   CPUSimulator::execute              CPUcode/simulator.hpp:71-128
//   exportqcx                          backendagnosticcode/Circuit.hpp:763-774
//   print                              backendagnosticcode/QuantumCircuit.hpp:38-123
//
// Thread-count pin: CPUSimulator::executeCommand splits 2^(n-14) groups over
// std::thread::hardware_concurrency() threads and silently drops the
// remainder (CPUcode/simulator.hpp:280-287). libstdc++ answers
// hardware_concurrency() through get_nprocs(); libstdc++ is linked statically
// into this library and get_nprocs() below (hidden, so it binds locally)
// returns a power of two: KATE_REF_THREADS if set, else the largest power of
// two not above the machine's online CPU count.

// The session entry points below drive CPUSimulator's gate phase alone
// (initialise once, then executeCommand per compute instruction, no
// measurement), which needs its private members; the reference sources are
// not modified.
// Standard headers first, so that only the reference's own classes see it.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits.h>
#include <list>
#include <math.h>
#include <queue>
#include <set>
#include <stdlib.h>
#include <string>
#include <thread>
#include <vector>
#define private public
#include "Kate.hpp"
#undef private

#include <sys/sysinfo.h>
#include <unistd.h>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>

extern "C" __attribute__((visibility("hidden"))) int get_nprocs(void) {
    const char* env = std::getenv("KATE_REF_THREADS");
    long n = 0;
    if (env && *env) n = std::strtol(env, nullptr, 10);
    if (n <= 0) n = sysconf(_SC_NPROCESSORS_ONLN);
    if (n <= 0) n = 1;
    long p = 1;
    while (p * 2 <= n) p *= 2;
    return (int)p;
}

namespace {

struct Handle {
    Kate::Circuit circ;
    explicit Handle(int n) : circ(n) {}
};

Kate::Gate make_gate(int id, int nq, const int* qbits, int optarg, const double* dense) {
    std::vector<int> q(qbits, qbits + nq);
    if (id == 0) {
        int dim = 1 << nq;
        Kate::Matrix<Kate::Complex> m(dim);
        for (int i = 0; i < dim * dim; i++) m.data[i] = Kate::Complex(dense[2 * i], dense[2 * i + 1]);
        return Kate::Gate(m, q);
    }
    return Kate::Gate(id, q, optarg);
}

}  // namespace

extern "C" {

int kref_hw_threads(void) { return (int)std::thread::hardware_concurrency(); }

void* kref_circuit_new(int n) { return new Handle(n); }
void kref_free(void* h) { delete static_cast<Handle*>(h); }

void kref_append(void* h, int id, int nq, const int* qbits, int optarg, const double* dense) {
    static_cast<Handle*>(h)->circ.appendGate(make_gate(id, nq, qbits, optarg, dense));
}

void kref_schedule(void* h) { static_cast<Handle*>(h)->circ.gateScheduling(); }
void kref_fuse(void* h, int k, double mtm) { static_cast<Handle*>(h)->circ.gateFusion(k, mtm); }
void kref_group(void* h, int m) { static_cast<Handle*>(h)->circ.gateGrouping(m); }
void kref_allocate(void* h, int g, int maxlocal) { static_cast<Handle*>(h)->circ.allocate(g, maxlocal); }
void kref_compile_default(void* h, int g, int maxlocal) {
    static_cast<Handle*>(h)->circ.compileDefault(g, maxlocal);
}

int kref_ngates(void* h) { return (int)static_cast<Handle*>(h)->circ.gate_set_ordered.size(); }

// Copies gate i out. dense (nullable) receives 2*4^nq doubles when id == 0.
void kref_gate(void* h, int i, int* id, int* nq, int* qbits, int* optarg, double* dense) {
    Kate::Gate& g = static_cast<Handle*>(h)->circ.gate_set_ordered[i];
    *id = g.identifier;
    *nq = (int)g.qbits.size();
    for (size_t k = 0; k < g.qbits.size(); k++) qbits[k] = g.qbits[k];
    *optarg = g.optarg;
    if (dense && g.identifier == 0) {
        int dim = g.densecontent.n;
        for (int k = 0; k < dim * dim; k++) {
            dense[2 * k] = g.densecontent.data[k].a;
            dense[2 * k + 1] = g.densecontent.data[k].b;
        }
    }
}

int kref_ngroups(void* h) { return (int)static_cast<Handle*>(h)->circ.groups.size(); }

void kref_group_get(void* h, int i, int* end, int* nq, int* qbits) {
    auto& g = static_cast<Handle*>(h)->circ.groups[i];
    *end = g.first;
    *nq = (int)g.second.size();
    int k = 0;
    for (int q : g.second) qbits[k++] = q;
}

int kref_ninstr(void* h) { return (int)static_cast<Handle*>(h)->circ.instructions.size(); }

void kref_instr(void* h, int i, int* kind, int* nq, int* qbits) {
    auto& ins = static_cast<Handle*>(h)->circ.instructions[i];
    *kind = ins.first;
    *nq = (int)ins.second.size();
    for (size_t k = 0; k < ins.second.size(); k++) qbits[k] = ins.second[k];
}

// init / final_inv receive nqbits ints each (left untouched when empty).
int kref_perms(void* h, int* init, int* final_inv) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    if (c.initial_permutation.size() != (size_t)c.nqbits) return 0;
    for (int i = 0; i < c.nqbits; i++) {
        init[i] = c.initial_permutation[i];
        final_inv[i] = c.final_inverse_permutation[i];
    }
    return 1;
}

// Merges gates [b, e) of the circuit with the reference's CPU merger.
// out_dense receives 2*4^k doubles; out_qbits k ints; returns k.
int kref_merge(void* h, int b, int e, int* out_qbits, double* out_dense) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    std::vector<Kate::Gate> to_merge(c.gate_set_ordered.begin() + b, c.gate_set_ordered.begin() + e);
    Kate::Gate g = Kate::mergeGate(to_merge);
    int k = (int)g.qbits.size();
    for (int i = 0; i < k; i++) out_qbits[i] = g.qbits[i];
    int dim = g.densecontent.n;
    for (int i = 0; i < dim * dim; i++) {
        out_dense[2 * i] = g.densecontent.data[i].a;
        out_dense[2 * i + 1] = g.densecontent.data[i].b;
    }
    return k;
}

// Runs the reference CPUSimulator on the circuit as it stands (it compiles
// naively if no instructions exist, as the reference does). state_out
// (nullable) receives 2*2^n doubles in the simulator's own amplitude order;
// proba_out (nullable) 2*n doubles (theta, phi per qubit); ms_out (nullable)
// the wall time of execute() in milliseconds. proba_in (nullable) selects
// execute(proba_state&).
int kref_simulate(void* h, const double* proba_in, double* state_out, double* proba_out, double* ms_out) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    Kate::Simulator sim(c, 0);
    int n = c.nqbits;
    auto t0 = std::chrono::steady_clock::now();
    Kate::proba_state res(n);
    if (proba_in) {
        Kate::proba_state in(n);
        for (int i = 0; i < n; i++) in.val[i] = std::make_pair(proba_in[2 * i], proba_in[2 * i + 1]);
        res = sim.execute(in, false);
    } else {
        res = sim.execute(false);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (ms_out) *ms_out = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (state_out) {
        size_t dim = (size_t)1 << n;
        for (size_t i = 0; i < dim; i++) {
            state_out[2 * i] = sim.qbitstate[i].a;
            state_out[2 * i + 1] = sim.qbitstate[i].b;
        }
    }
    if (proba_out) {
        for (int i = 0; i < n; i++) {
            proba_out[2 * i] = res.val[i].first;
            proba_out[2 * i + 1] = res.val[i].second;
        }
    }
    return 0;
}

// Gate-phase timing session: a CPUSimulator on the circuit as it stands,
// initialised once to |0..0>; each kref_session_run executes every compute
// instruction once more (CPUcode/simulator.hpp:76-84) and returns its wall
// time in ms. The state keeps evolving across runs.
void* kref_session_new(void* h) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    auto* sim = new Kate::Simulator(c, 0);
    if (!sim->qbitstate) {
        delete sim;
        return nullptr;
    }
    sim->initialize();
    return sim;
}

double kref_session_run(void* s) {
    auto* sim = static_cast<Kate::Simulator*>(s);
    auto t0 = std::chrono::steady_clock::now();
    int groupid = 0;
    for (const auto& instr : sim->instructions) {
        if (instr.first == 1) {
            sim->executeCommand(groupid);
            groupid++;
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

void kref_session_free(void* s) { delete static_cast<Kate::Simulator*>(s); }

void kref_export_qcx(void* h, const char* path) { static_cast<Handle*>(h)->circ.exportqcx(std::string(path)); }

// QuantumCircuit::print(permutationtable) with std::cout appended to `path`.
int kref_print(void* h, int permutationtable, const char* path) {
    std::ofstream f(path, std::ios::app);
    if (!f) return 1;
    std::streambuf* old = std::cout.rdbuf(f.rdbuf());
    static_cast<Handle*>(h)->circ.print(permutationtable != 0);
    std::cout.flush();
    std::cout.rdbuf(old);
    return 0;
}

}  // extern "C"
