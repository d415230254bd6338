// Measurement reductions over the state, FP64 accumulation.
//
// k_bitsums computes, for every bit b of the amplitude index, the sum over
// amplitudes whose bit b is 0 and the sum over those whose bit b is 1 (kind
// 0: the amplitudes themselves, the reference's proba_state input,
// HIPcode/simulator.hpp:40-61 and 483-543; kind 1: |a|^2, for <Z_q>), in one
// read pass. Element x is split as
//   x = ((r << g) | cta) << 12 | j << 8 | t
// (t = thread, j = 0..15 unrolled, cta = blockIdx, r = round). The sums over
// t-bits and j-bits are exact subset sums of per-thread accumulators; the
// cta-bits are resolved on the host from per-CTA totals; r-bits are
// accumulated per thread. Each CTA writes its partials; the host adds them
// in CTA order (deterministic).
#include "k_common.cuh"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NT = 256;
constexpr int MAXR = 8;

template <typename V>
struct Acc;
template <>
struct Acc<double2> {
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 val(double2 a) { return a; }
    __device__ static double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
    __device__ static double2 shfl(double2 v, int o) {
        return make_double2(__shfl_down_sync(0xffffffffu, v.x, o), __shfl_down_sync(0xffffffffu, v.y, o));
    }
};
template <>
struct Acc<double> {
    __device__ static double zero() { return 0.0; }
    __device__ static double val(double2 a) { return a.x * a.x + a.y * a.y; }
    __device__ static double add(double a, double b) { return a + b; }
    __device__ static double shfl(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
};

// Output slots per CTA: 0 = total; 1 + 2*b = bit b is 0; 2 + 2*b = bit b is
// 1, for local bits b = 0..11 then round bits 12..12+nr-1 (numbered in slot
// order, not in index order).
__device__ __forceinline__ double2 ld_amp(const double2* p) { return *p; }
__device__ __forceinline__ double2 ld_amp(const float2* p) {
    const float2 v = *p;
    return make_double2(v.x, v.y);
}

// S: stored amplitude type (double2 or float2); sums are FP64 either way.
template <typename V, typename S = double2>
__global__ void __launch_bounds__(NT, 2) k_bitsums(const S* __restrict__ st, int n, int g, int nr,
                                                V* __restrict__ part) {
    using A = Acc<V>;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int lb = n < 12 ? n : 12;
    const uint32_t lim = 1u << lb;
    V T = A::zero(), H0[4], H1[4], R0[MAXR], R1[MAXR];
#pragma unroll
    for (int i = 0; i < 4; i++) H0[i] = H1[i] = A::zero();
#pragma unroll
    for (int i = 0; i < MAXR; i++) R0[i] = R1[i] = A::zero();
    const uint64_t rounds = 1ull << nr;
    for (uint64_t r = 0; r < rounds; r++) {
        const uint64_t base = ((r << g) | blockIdx.x) << 12;
        V tr = A::zero();
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t x = (uint32_t)t + ((uint32_t)j << 8);
            V v = A::zero();
            if (x < lim) v = A::val(ld_amp(st + base + x));
            tr = A::add(tr, v);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if ((j >> i) & 1) H1[i] = A::add(H1[i], v);
                else H0[i] = A::add(H0[i], v);
            }
        }
        T = A::add(T, tr);
#pragma unroll
        for (int i = 0; i < MAXR; i++)
            if (i < nr) {
                if ((r >> i) & 1) R1[i] = A::add(R1[i], tr);
                else R0[i] = A::add(R0[i], tr);
            }
    }
    // Slots reduced per warp: 0 total; 1..5 lane-bit-1 sums; 6..10
    // lane-bit-0 sums; 11..14 H0; 15..18 H1; 19.. R0; 19+MAXR.. R1.
    constexpr int NS = 19 + 2 * MAXR;
    __shared__ V sm[NT / 32][NS];
    auto wsum = [&](V v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = A::add(v, A::shfl(v, o));
        return v;
    };
    V w;
    w = wsum(T);
    if (lane == 0) sm[warp][0] = w;
#pragma unroll
    for (int b = 0; b < 5; b++) {
        w = wsum(((lane >> b) & 1) ? T : A::zero());
        if (lane == 0) sm[warp][1 + b] = w;
        w = wsum(((lane >> b) & 1) ? A::zero() : T);
        if (lane == 0) sm[warp][6 + b] = w;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        w = wsum(H0[i]);
        if (lane == 0) sm[warp][11 + i] = w;
        w = wsum(H1[i]);
        if (lane == 0) sm[warp][15 + i] = w;
    }
#pragma unroll
    for (int i = 0; i < MAXR; i++) {
        if (i < nr) {
            w = wsum(R0[i]);
            if (lane == 0) sm[warp][19 + i] = w;
            w = wsum(R1[i]);
            if (lane == 0) sm[warp][19 + MAXR + i] = w;
        }
    }
    __syncthreads();
    const int nout = 1 + 2 * (12 + nr);
    if (t < nout) {
        V s = A::zero();
        if (t == 0) {
            for (int ww = 0; ww < NT / 32; ww++) s = A::add(s, sm[ww][0]);
        } else {
            const int b = (t - 1) / 2, one = (t - 1) & 1;
            for (int ww = 0; ww < NT / 32; ww++) {
                V v;
                if (b < 5) v = one ? sm[ww][1 + b] : sm[ww][6 + b];
                else if (b < 8) v = (((ww >> (b - 5)) & 1) == one) ? sm[ww][0] : A::zero();
                else if (b < 12) v = one ? sm[ww][15 + (b - 8)] : sm[ww][11 + (b - 8)];
                else v = one ? sm[ww][19 + MAXR + (b - 12)] : sm[ww][19 + (b - 12)];
                s = A::add(s, v);
            }
        }
        part[(size_t)blockIdx.x * nout + t] = s;
    }
}

template <typename S>
__global__ void k_probs(const S* __restrict__ st, uint64_t dim, double* __restrict__ out) {
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
        const double2 a = ld_amp(st + x);
        out[x] = a.x * a.x + a.y * a.y;
    }
}

// ---- renormalisation of complex64 states ----
// ||psi||^2 in FP64: each CTA sums |a|^2 over a grid-stride range (16-byte
// loads, two amplitudes each, in a fixed per-thread order), reduces it in a
// fixed tree, writes its partial; the last CTA to finish adds the partials
// in CTA order (deterministic) and writes out[0] = ||psi||^2 and out[1] =
// 1 / ||psi||, then resets the counter for the next run.
constexpr int RN_GRID = 148 * 4;

__global__ void __launch_bounds__(256) k_norm2_c64(const float4* __restrict__ st, uint64_t npairs,
                                                   double* __restrict__ part, unsigned* __restrict__ count,
                                                   double* __restrict__ out) {
    __shared__ double red[256];
    __shared__ bool last;
    const uint32_t t = threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    double acc = 0.0;
    uint64_t i = (uint64_t)blockIdx.x * 256 + t;
    for (; i + 3 * stride < npairs; i += 4 * stride) {
        float4 v[4];
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = __ldcs(st + i + k * stride);
#pragma unroll
        for (int k = 0; k < 4; k++)
            acc += ((double)v[k].x * v[k].x + (double)v[k].y * v[k].y) + ((double)v[k].z * v[k].z + (double)v[k].w * v[k].w);
    }
    for (; i < npairs; i += stride) {
        const float4 v = __ldcs(st + i);
        acc += ((double)v.x * v.x + (double)v.y * v.y) + ((double)v.z * v.z + (double)v.w * v.w);
    }
    red[t] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < (uint32_t)w) red[t] += red[t + w];
        __syncthreads();
    }
    if (t == 0) {
        part[blockIdx.x] = red[0];
        __threadfence();
        last = atomicAdd(count, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && t == 0) {
        __threadfence();
        double tot = 0.0;
        for (uint32_t c = 0; c < gridDim.x; c++) tot += ((volatile double*)part)[c];
        out[0] = tot;
        out[1] = tot > 0.0 ? 1.0 / sqrt(tot) : 1.0;
        *count = 0;
    }
}

// Multiplies every amplitude by the scale the norm kernel wrote (read on
// the device: no host round trip between the two launches). The product is
// formed in FP64 and rounded once, so each amplitude carries only its own
// rounding error; a scale rounded to FP32 first would shift the whole norm
// by up to 2^-23.
__global__ void __launch_bounds__(256) k_scale_c64(float4* __restrict__ st, uint64_t npairs,
                                                   const double* __restrict__ out) {
    const double f = out[1];
    const uint64_t stride = (uint64_t)gridDim.x * 256;
    for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < npairs; i += stride) {
        float4 v = __ldcs(st + i);
        v.x = (float)((double)v.x * f);
        v.y = (float)((double)v.y * f);
        v.z = (float)((double)v.z * f);
        v.w = (float)((double)v.w * f);
        __stcs(st + i, v);
    }
}

}  // namespace

size_t renorm_scratch_bytes() { return (RN_GRID + 4) * sizeof(double); }

cudaError_t launch_renorm_c64(void* st, int n, void* scratch, cudaStream_t s) {
    if (n < 1) return cudaErrorInvalidValue;
    const uint64_t npairs = (1ull << n) / 2;
    double* part = (double*)scratch;
    double* out = part + RN_GRID;
    unsigned* count = (unsigned*)(out + 2);
    const unsigned grid = (unsigned)(npairs < (uint64_t)RN_GRID * 256 ? (npairs + 255) / 256 : RN_GRID);
    k_norm2_c64<<<grid, 256, 0, s>>>((const float4*)st, npairs, part, count, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_scale_c64<<<grid, 256, 0, s>>>((float4*)st, npairs, out);
    return cudaGetLastError();
}

BitSumShape bitsum_shape(int n) {
    BitSumShape s{};
    if (n <= 12) {
        s.g = 0;
        s.nr = 0;
    } else {
        // About a thousand CTAs (seven per SM), each summing up to 2^MAXR
        // rounds in registers: few partials to add on the host.
        s.g = n - 12 < 10 ? n - 12 : 10;
        s.nr = n - 12 - s.g;
        if (s.nr > MAXR) {
            s.nr = MAXR;
            s.g = n - 12 - MAXR;
        }
    }
    s.grid = 1 << s.g;
    s.nout = 1 + 2 * (12 + s.nr);
    return s;
}

cudaError_t launch_bitsums_c128(const void* st, int n, int kind, void* partials, cudaStream_t s) {
    BitSumShape sh = bitsum_shape(n);
    if (sh.nr > MAXR) return cudaErrorInvalidValue;
    if (kind == 0)
        k_bitsums<double2><<<sh.grid, NT, 0, s>>>((const double2*)st, n, sh.g, sh.nr, (double2*)partials);
    else
        k_bitsums<double><<<sh.grid, NT, 0, s>>>((const double2*)st, n, sh.g, sh.nr, (double*)partials);
    return cudaGetLastError();
}

cudaError_t launch_bitsums_c128_shape(const void* st, int n, int g, int nr, void* partials, cudaStream_t s) {
    if (nr < 0 || nr > MAXR || g < 0) return cudaErrorInvalidValue;
    k_bitsums<double2><<<1 << g, NT, 0, s>>>((const double2*)st, n, g, nr, (double2*)partials);
    return cudaGetLastError();
}

cudaError_t launch_probs_c128(const void* st, uint64_t dim, double* out, cudaStream_t s) {
    uint64_t blocks = (dim + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_probs<double2><<<(unsigned)blocks, 256, 0, s>>>((const double2*)st, dim, out);
    return cudaGetLastError();
}

cudaError_t launch_bitsums(const void* st, int prec, int n, int kind, void* partials, cudaStream_t s) {
    if (prec == 0) return launch_bitsums_c128(st, n, kind, partials, s);
    BitSumShape sh = bitsum_shape(n);
    if (sh.nr > MAXR) return cudaErrorInvalidValue;
    if (kind == 0)
        k_bitsums<double2, float2><<<sh.grid, NT, 0, s>>>((const float2*)st, n, sh.g, sh.nr, (double2*)partials);
    else
        k_bitsums<double, float2><<<sh.grid, NT, 0, s>>>((const float2*)st, n, sh.g, sh.nr, (double*)partials);
    return cudaGetLastError();
}

cudaError_t launch_probs(const void* st, int prec, uint64_t dim, double* out, cudaStream_t s) {
    if (prec == 0) return launch_probs_c128(st, dim, out, s);
    uint64_t blocks = (dim + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_probs<float2><<<(unsigned)blocks, 256, 0, s>>>((const float2*)st, dim, out);
    return cudaGetLastError();
}

}  // namespace kate
