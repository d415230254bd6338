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

__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ void narrow(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void narrow(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// A (global amplitude type): double2 for complex128 states, float2 for
// complex64; the shared-memory tile is double2 either way.
template <typename A>
__global__ void __launch_bounds__(NT) k_pass_generic(A* __restrict__ st, const DevPass P,
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
            tile[ops::swz(i)] = widen(st[a]);
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
            narrow(st + a, tile[ops::swz(i)]);
        }
        __syncthreads();
    }
}

template <typename A>
__global__ void k_set_one(A* st) {
    narrow(st, make_double2(1.0, 0.0));
}

template <typename A>
__global__ void k_init_product(A* __restrict__ st, int n, const ProductInit P) {
    const uint64_t dim = 1ull << n;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
        double2 t = make_double2(1.0, 0.0);
        for (int j = 0; j < n; j++) {
            int b = (int)((x >> j) & 1ull);
            t = cmul(t, make_double2(P.v[b][j][0], P.v[b][j][1]));
        }
        narrow(st + x, t);
    }
}

// The same product state for n >= 10 in one write pass: amplitude
// (c << 10) | i is L[i] * H(c), L the products of the low 10 qubits' factors
// (a shared table built once per CTA) and H the product of the high ones
// (per 1024-amplitude chunk, the same for the whole block, so its factor
// loads are uniform). The product is taken in another order than the
// reference's left-to-right one: the amplitudes agree to a few ulp.
template <typename A>
__global__ void __launch_bounds__(256) k_init_product_split(A* __restrict__ st, int n, const ProductInit P) {
    __shared__ double2 L[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) {
        double2 v = make_double2(1.0, 0.0);
        for (int j = 0; j < 10; j++) {
            const int b = (i >> j) & 1;
            v = cmul(v, make_double2(P.v[b][j][0], P.v[b][j][1]));
        }
        L[i] = v;
    }
    __syncthreads();
    const uint64_t nchunks = 1ull << (n - 10);
    for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        double2 h = make_double2(1.0, 0.0);
        for (int j = 10; j < n; j++) {
            const int b = (int)((c >> (j - 10)) & 1ull);
            h = cmul(h, make_double2(P.v[b][j][0], P.v[b][j][1]));
        }
        A* dst = st + (c << 10);
        for (int i = threadIdx.x; i < 1024; i += blockDim.x) narrow(dst + i, cmul(L[i], h));
    }
}

}  // namespace

cudaError_t launch_set_basis0(void* st, uint64_t dim, int prec, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(st, 0, dim * (prec == 0 ? sizeof(double2) : sizeof(float2)), s);
    if (e != cudaSuccess) return e;
    if (prec == 0) k_set_one<double2><<<1, 1, 0, s>>>((double2*)st);
    else k_set_one<float2><<<1, 1, 0, s>>>((float2*)st);
    return cudaGetLastError();
}

cudaError_t launch_set_basis0_c128(void* st, uint64_t dim, cudaStream_t s) { return launch_set_basis0(st, dim, 0, s); }

cudaError_t launch_init_product(void* st, int n, const ProductInit& P, int prec, cudaStream_t s) {
    if (n >= 10) {
        const uint64_t nchunks = 1ull << (n - 10);
        const unsigned blocks = (unsigned)(nchunks < 148 * 8 ? nchunks : 148 * 8);
        if (prec == 0) k_init_product_split<double2><<<blocks, 256, 0, s>>>((double2*)st, n, P);
        else k_init_product_split<float2><<<blocks, 256, 0, s>>>((float2*)st, n, P);
        return cudaGetLastError();
    }
    uint64_t dim = 1ull << n;
    uint64_t blocks = (dim + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (prec == 0) k_init_product<double2><<<(unsigned)blocks, 256, 0, s>>>((double2*)st, n, P);
    else k_init_product<float2><<<(unsigned)blocks, 256, 0, s>>>((float2*)st, n, P);
    return cudaGetLastError();
}

cudaError_t launch_init_product_c128(void* st, int n, const ProductInit& P, cudaStream_t s) {
    return launch_init_product(st, n, P, 0, s);
}

int generic_pass_grid(int n, int m, int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        const int smem = (1 << MAXM) * (int)sizeof(double2);
        cudaFuncSetAttribute(k_pass_generic<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_pass_generic<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pass_generic<double2>, NT, smem);
        if (occ < 1) occ = 1;
        cached[device] = sms * occ;
    }
    uint64_t ncos = 1ull << (n - m);
    return (int)(ncos < (uint64_t)cached[device] ? ncos : (uint64_t)cached[device]);
}

cudaError_t launch_pass_generic(void* st, int prec, const DevPass& p, const DevOp* ops, const void* pool, int grid,
                                cudaStream_t s) {
    if (p.m > MAXM) return cudaErrorInvalidValue;
    size_t smem = ((size_t)1 << p.m) * sizeof(double2);
    if (prec == 0) k_pass_generic<double2><<<grid, NT, smem, s>>>((double2*)st, p, ops, (const double2*)pool);
    else k_pass_generic<float2><<<grid, NT, smem, s>>>((float2*)st, p, ops, (const double2*)pool);
    return cudaGetLastError();
}

cudaError_t launch_pass_generic_c128(void* st, int n, const DevPass& p, const DevOp* ops, const void* pool, int grid,
                                     cudaStream_t s) {
    (void)n;
    return launch_pass_generic(st, 0, p, ops, pool, grid, s);
}

}  // namespace kate
