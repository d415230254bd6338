// Inverse-CDF sampling of the computational basis on the device, for the
// simulator (kate_sim_sample), without copying the probabilities to the
// host: only the shots' uniforms go to the device and the sampled indices
// come back.
//
// Shot s with uniform u_s in [0, 1) (ascending on the device; the host keeps
// the draw order) takes the first amplitude index i whose cumulative
// probability exceeds y_s = u_s * total, i.e. cdf(i - 1) <= y_s < cdf(i);
// amplitudes of probability 0 are never chosen. The cumulative sums are FP64
// and fixed-order:
//   k_chunk_sums  sum of |a|^2 over each chunk of 2^16 amplitudes (a block
//                 reduction in a fixed tree);
//   k_chunk_scan  exclusive prefix of the chunk sums and their total (one
//                 CTA, a fixed order);
//   k_resolve     one CTA per chunk: the shots whose target falls in the
//                 chunk (a binary search over the sorted uniforms), then a
//                 block scan over per-thread runs of 256 amplitudes locates
//                 each target's run, whose thread walks it.
// Indices are physical (the state's bit layout); the host maps them to the
// reference's qubit labels. This is the device counterpart of the
// reference's host-side measurement (HIPcode/simulator.hpp:483-543 copies
// partial sums back); Kate itself has no sampling.
#include "k_common.cuh"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NTS = 256;
constexpr int CHUNK_BITS = 16;

__device__ __forceinline__ double prob(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double prob(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }

// Fixed-order block sum of one double per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* red) {
    const uint32_t t = threadIdx.x;
    red[t] = v;
    __syncthreads();
    for (int w = NTS / 2; w > 0; w >>= 1) {
        if (t < (uint32_t)w) red[t] += red[t + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// Fixed-order block exclusive scan of one double per thread; *total gets
// the block total.
__device__ __forceinline__ double block_exscan(double v, double* red, double* total) {
    const uint32_t t = threadIdx.x;
    red[t] = v;
    __syncthreads();
    if (t == 0) {
        double run = 0.0;
        for (int i = 0; i < NTS; i++) {
            const double x = red[i];
            red[i] = run;
            run += x;
        }
        red[NTS] = run;
    }
    __syncthreads();
    const double r = red[t];
    *total = red[NTS];
    __syncthreads();
    return r;
}

template <typename C2>
__global__ void __launch_bounds__(NTS) k_chunk_sums(const C2* __restrict__ st, int n, double* __restrict__ sums) {
    __shared__ double red[NTS + 1];
    const uint64_t dim = 1ull << n;
    const uint64_t x0 = (uint64_t)blockIdx.x << CHUNK_BITS;
    double acc = 0.0;
    for (uint32_t k = 0; k < (1u << CHUNK_BITS) / NTS; k++) {
        const uint64_t x = x0 + ((uint64_t)k * NTS) + threadIdx.x;
        if (x < dim) acc += prob(st[x]);
    }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

// pre[c] = sum of sums[0..c), pre[nch] = total. One CTA of 1024 threads,
// each owning a contiguous run of chunks.
__global__ void __launch_bounds__(1024) k_chunk_scan(const double* __restrict__ sums, uint32_t nch,
                                                     double* __restrict__ pre) {
    __shared__ double part[1025];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (nch + 1023) / 1024, b0 = t * per, b1 = min(nch, b0 + per);
    double loc = 0.0;
    for (uint32_t c = b0; c < b1; c++) loc += sums[c];
    part[t] = loc;
    __syncthreads();
    if (t == 0) {
        double run = 0.0;
        for (int i = 0; i < 1024; i++) {
            const double x = part[i];
            part[i] = run;
            run += x;
        }
        part[1024] = run;
    }
    __syncthreads();
    double run = part[t];
    for (uint32_t c = b0; c < b1; c++) {
        pre[c] = run;
        run += sums[c];
    }
    if (t == 0) pre[nch] = part[1024];
}

// First index s in [0, shots) with unif[s] * total >= v (shots if none).
__device__ __forceinline__ int first_at_least(const double* unif, int shots, double total, double v) {
    int lo = 0, hi = shots;
    while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (unif[m] * total >= v) hi = m;
        else lo = m + 1;
    }
    return lo;
}

template <typename C2>
__global__ void __launch_bounds__(NTS) k_resolve(const C2* __restrict__ st, int n, const double* __restrict__ pre,
                                                 uint32_t nch, const double* __restrict__ unif, int shots,
                                                 uint64_t* __restrict__ out) {
    __shared__ double red[NTS + 1];
    __shared__ int range[2];
    const uint32_t ch = blockIdx.x, t = threadIdx.x;
    const double total = pre[nch];
    const double lo_v = pre[ch], hi_v = pre[ch + 1];
    const bool last = ch + 1 == nch;
    if (t == 0) {
        // Targets y in [lo_v, hi_v) fall here; the last chunk also takes
        // targets at or past the total (rounding).
        range[0] = ch == 0 ? 0 : first_at_least(unif, shots, total, lo_v);
        range[1] = last ? shots : first_at_least(unif, shots, total, hi_v);
    }
    __syncthreads();
    const int s0 = range[0], s1 = range[1];
    if (s0 >= s1) return;
    const uint64_t dim = 1ull << n;
    const uint64_t x0 = (uint64_t)ch << CHUNK_BITS;
    const uint64_t len = dim - x0 < (1ull << CHUNK_BITS) ? dim - x0 : (1ull << CHUNK_BITS);
    const uint64_t per = (len + NTS - 1) / NTS;
    const uint64_t a0 = x0 + min((uint64_t)t * per, len), a1 = x0 + min((uint64_t)(t + 1) * per, len);
    double w = 0.0;
    for (uint64_t x = a0; x < a1; x++) w += prob(st[x]);
    double btot;
    const double base = block_exscan(w, red, &btot);
    // The run holding target y: base <= y < base + w. Targets past the
    // chunk's last run (rounding between the chunk sum and the runs) go to
    // the last non-empty amplitude of the chunk.
    for (int s = s0 + (int)t; s < s1; s += NTS) {
        // Every thread resolves its own shots: find the run by a binary
        // search over the runs' bases (kept in red[0..NTS)).
        const double y = unif[s] * total - lo_v;
        int lo = 0, hi = NTS - 1;  // last run with base <= y
        while (lo < hi) {
            const int m = (lo + hi + 1) >> 1;
            if (red[m] <= y) lo = m;
            else hi = m - 1;
        }
        const uint64_t r0 = x0 + min((uint64_t)lo * per, len), r1 = x0 + min((uint64_t)(lo + 1) * per, len);
        double c = red[lo];
        uint64_t pick = r1 > r0 ? r1 - 1 : x0;
        uint64_t lastnz = (uint64_t)-1;
        for (uint64_t x = r0; x < r1; x++) {
            const double p = prob(st[x]);
            if (p > 0.0) lastnz = x;
            c += p;
            if (c > y && p > 0.0) {
                pick = x;
                lastnz = (uint64_t)-2;
                break;
            }
        }
        if (lastnz != (uint64_t)-2) {
            // y at or past the run's end: the last amplitude of nonzero
            // probability at or before it in the chunk.
            if (lastnz != (uint64_t)-1) pick = lastnz;
            else
                for (uint64_t x = r0; x-- > x0;)
                    if (prob(st[x]) > 0.0) {
                        pick = x;
                        break;
                    }
        }
        out[s] = pick;
    }
}

}  // namespace

size_t sample_scratch_doubles(int n) {
    const uint32_t nch = n > CHUNK_BITS ? 1u << (n - CHUNK_BITS) : 1u;
    return 2 * (size_t)nch + 1;
}

cudaError_t launch_sample(const void* st, int prec, int n, const double* unif, int shots, double* scratch,
                          uint64_t* out, cudaStream_t s) {
    if (n < 1 || shots < 0) return cudaErrorInvalidValue;
    const uint32_t nch = n > CHUNK_BITS ? 1u << (n - CHUNK_BITS) : 1u;
    double* sums = scratch;
    double* pre = scratch + nch;
    if (prec == 1) k_chunk_sums<float2><<<nch, NTS, 0, s>>>((const float2*)st, n, sums);
    else k_chunk_sums<double2><<<nch, NTS, 0, s>>>((const double2*)st, n, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_chunk_scan<<<1, 1024, 0, s>>>(sums, nch, pre);
    e = cudaGetLastError();
    if (e != cudaSuccess || shots == 0) return e;
    if (prec == 1) k_resolve<float2><<<nch, NTS, 0, s>>>((const float2*)st, n, pre, nch, unif, shots, out);
    else k_resolve<double2><<<nch, NTS, 0, s>>>((const double2*)st, n, pre, nch, unif, shots, out);
    return cudaGetLastError();
}

}  // namespace kate
