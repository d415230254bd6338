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
#include "k_ops.cuh"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NT = 256;
constexpr int MAXM = 12;

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
            tile[ops::swz(i)] = st[a];
        }
        __syncthreads();
        for (int k = 0; k < P.nops; k++) {
            const DevOp op = ops[P.op0 + k];
            ops::apply_op(tile, m, base, op, pool, threadIdx.x, NT);
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
            st[a] = tile[ops::swz(i)];
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
