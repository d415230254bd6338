// Generic complex128 group-pass kernel and state initialisation.
//
// One CTA per coset of the pass's tile: the 2^m amplitudes that share all
// non-tile bits are gathered into shared memory (every run of 2^c low
// physical bits is contiguous, so each warp load covers whole 128-byte
// lines), every op of the pass is applied in shared memory, and the tile is
// written back with its tile bits permuted by `outsrc` (the qubit remap).
// This is the replacement for the reference's executeGroupKernelSharedState
// + GPUGate::compute (HIPcode/simulator.hpp:143-218, HIPcode/GPUGate.hpp:21-203)
// and handles every op kind, including dense blocks of up to 5 qubits.
#include "k_common.cuh"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NT = 256;
constexpr int MAXM = 12;

template <int K>
__device__ void op_dense(double2* s, int m, const DevOp& op, const double2* __restrict__ mat) {
    constexpr int D = 1 << K;
    int tb[K], srt[K];
#pragma unroll
    for (int i = 0; i < K; i++) tb[i] = srt[i] = op.tb[i];
#pragma unroll
    for (int i = 1; i < K; i++)
#pragma unroll
        for (int j = K - 1; j >= i; j--)
            if (srt[j - 1] > srt[j]) {
                int t = srt[j];
                srt[j] = srt[j - 1];
                srt[j - 1] = t;
            }
    const uint32_t groups = 1u << (m - K);
    for (uint32_t g = threadIdx.x; g < groups; g += NT) {
        uint32_t base = g;
#pragma unroll
        for (int i = 0; i < K; i++) base = ins0(base, srt[i]);
        double2 x[D];
#pragma unroll
        for (int v = 0; v < D; v++) {
            uint32_t idx = base;
#pragma unroll
            for (int i = 0; i < K; i++)
                if ((v >> i) & 1) idx |= 1u << tb[i];
            x[v] = s[idx];
        }
#pragma unroll
        for (int r = 0; r < D; r++) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < D; c++) cfma(acc, __ldg(mat + r * D + c), x[c]);
            uint32_t idx = base;
#pragma unroll
            for (int i = 0; i < K; i++)
                if ((r >> i) & 1) idx |= 1u << tb[i];
            s[idx] = acc;
        }
    }
}

__device__ void apply_op(double2* s, int m, uint64_t base, const DevOp& op, const double2* __restrict__ pool) {
    const uint32_t T = 1u << m;
    switch (op.kind) {
    case OPK_H: {
        const int t = op.tb[0];
        for (uint32_t p = threadIdx.x; p < T / 2; p += NT) {
            uint32_t i0 = ins0(p, t), i1 = i0 | (1u << t);
            double2 a = s[i0], b = s[i1];
            double2 n0 = make_double2((a.x + b.x) * KATE_SQRT2INV, (a.y + b.y) * KATE_SQRT2INV);
            s[i0] = n0;
            s[i1] = make_double2(n0.x - b.x * KATE_SQRT2, n0.y - b.y * KATE_SQRT2);
        }
        break;
    }
    case OPK_X: {
        if ((base & op.pmask) != op.pmask) break;
        const int t = op.tb[0];
        for (uint32_t p = threadIdx.x; p < T / 2; p += NT) {
            uint32_t i0 = ins0(p, t);
            if ((i0 & op.tmask) != op.tmask) continue;
            uint32_t i1 = i0 | (1u << t);
            double2 a = s[i0];
            s[i0] = s[i1];
            s[i1] = a;
        }
        break;
    }
    case OPK_PHASE: {
        if ((base & op.pmask) != op.pmask) break;
        const double2 ph = make_double2(op.ph_re, op.ph_im);
        for (uint32_t i = threadIdx.x; i < T; i += NT)
            if ((i & op.tmask) == op.tmask) s[i] = cmul(s[i], ph);
        break;
    }
    case OPK_DIAG: {
        uint32_t cidx = 0;
        for (int i = 0; i < op.k; i++)
            if (op.ftb[i] < 0) cidx |= (uint32_t)((base >> op.fpos[i]) & 1ull) << i;
        const double2* tab = pool + op.mat;
        for (uint32_t x = threadIdx.x; x < T; x += NT) {
            uint32_t d = cidx;
            for (int i = 0; i < op.k; i++)
                if (op.ftb[i] >= 0) d |= ((x >> op.ftb[i]) & 1u) << i;
            s[x] = cmul(s[x], __ldg(tab + d));
        }
        break;
    }
    case OPK_DENSE: {
        const double2* mat = pool + op.mat;
        switch (op.k) {
        case 1: op_dense<1>(s, m, op, mat); break;
        case 2: op_dense<2>(s, m, op, mat); break;
        case 3: op_dense<3>(s, m, op, mat); break;
        case 4: op_dense<4>(s, m, op, mat); break;
        case 5: op_dense<5>(s, m, op, mat); break;
        default: break;
        }
        break;
    }
    default:
        break;
    }
}

__global__ void __launch_bounds__(NT) k_pass_generic(double2* __restrict__ st, const DevPass P,
                                                     const DevOp* __restrict__ ops,
                                                     const double2* __restrict__ pool) {
    extern __shared__ double2 tile[];
    const int m = P.m;
    const uint32_t T = 1u << m;
    const uint64_t ncos = 1ull << P.ncb;
    for (uint64_t c = blockIdx.x; c < ncos; c += gridDim.x) {
        uint64_t base = 0;
        for (int i = 0; i < P.ncb; i++) base |= ((c >> i) & 1ull) << P.cphys[i];
        for (uint32_t i = threadIdx.x; i < T; i += NT) {
            uint64_t a = base;
            for (int b = 0; b < m; b++) a |= (uint64_t)((i >> b) & 1u) << P.tphys[b];
            tile[i] = st[a];
        }
        __syncthreads();
        for (int k = 0; k < P.nops; k++) {
            const DevOp op = ops[P.op0 + k];
            apply_op(tile, m, base, op, pool);
            __syncthreads();
        }
        for (uint32_t o = threadIdx.x; o < T; o += NT) {
            uint64_t a = base;
            uint32_t i = 0;
            for (int b = 0; b < m; b++) {
                uint32_t bit = (o >> b) & 1u;
                a |= (uint64_t)bit << P.tphys[b];
                i |= bit << P.outsrc[b];
            }
            st[a] = tile[i];
        }
        __syncthreads();
    }
}

__global__ void k_set_one(double2* st) { st[0] = make_double2(1.0, 0.0); }

__global__ void k_init_product(double2* __restrict__ st, int n, const ProductInit P) {
    const uint64_t dim = 1ull << n;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
        double2 t = make_double2(1.0, 0.0);
        for (int j = 0; j < n; j++) {
            int b = (int)((x >> j) & 1ull);
            t = cmul(t, make_double2(P.v[b][j][0], P.v[b][j][1]));
        }
        st[x] = t;
    }
}

}  // namespace

cudaError_t launch_set_basis0_c128(void* st, uint64_t dim, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(st, 0, dim * sizeof(double2), s);
    if (e != cudaSuccess) return e;
    k_set_one<<<1, 1, 0, s>>>((double2*)st);
    return cudaGetLastError();
}

cudaError_t launch_init_product_c128(void* st, int n, const ProductInit& P, cudaStream_t s) {
    uint64_t dim = 1ull << n;
    uint64_t blocks = (dim + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_init_product<<<(unsigned)blocks, 256, 0, s>>>((double2*)st, n, P);
    return cudaGetLastError();
}

int generic_pass_grid(int n, int m, int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        cudaFuncSetAttribute(k_pass_generic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (1 << MAXM) * (int)sizeof(double2));
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pass_generic, NT, (1 << MAXM) * sizeof(double2));
        if (occ < 1) occ = 1;
        cached[device] = sms * occ;
    }
    uint64_t ncos = 1ull << (n - m);
    return (int)(ncos < (uint64_t)cached[device] ? ncos : (uint64_t)cached[device]);
}

cudaError_t launch_pass_generic_c128(void* st, int n, const DevPass& p, const DevOp* ops, const void* pool, int grid,
                                     cudaStream_t s) {
    (void)n;
    if (p.m > MAXM) return cudaErrorInvalidValue;
    size_t smem = ((size_t)1 << p.m) * sizeof(double2);
    k_pass_generic<<<grid, NT, smem, s>>>((double2*)st, p, ops, (const double2*)pool);
    return cudaGetLastError();
}

}  // namespace kate
