// Complex64 group pass with 5-qubit dense blocks on the tensor cores
// (tcgen05, kind::tf32, 3xTF32 compensated products, FP32 accumulation in
// TMEM).
//
// Each CTA (256 threads, one per SM) processes 4096-amplitude coset tiles
// in a grid-stride loop; the next tile is prefetched with cp.async into a
// second staging buffer while the current one is processed. For each block
// of the pass:
//   1. the tile (staging buffer S, natural tile order) is rearranged into
//      the MMA A operand: 128 rows (the values of the 7 non-block tile
//      bits) x 64 reals (the 32 complex amplitudes of the block's index,
//      re/im interleaved), K-major with the 128-byte swizzle, as a TF32 hi
//      part and the FP32 remainder (lo);
//   2. one elected thread issues 8 K-steps x 3 products (A_hi.B_hi,
//      A_hi.B_lo, A_lo.B_hi; M = 128, N = 64, K = 8) into one TMEM
//      accumulator and commits to an mbarrier;
//   3. every thread reads its row's 32 results back from TMEM and writes
//      them to S at the amplitudes' tile positions.
// The tile is then written back to global with the pass's remap permutation.
// The block matrices (B operands, hi and lo) are staged in shared memory
// once per CTA. All waits are bounded: on timeout the kernel records an
// error flag for the host and returns after freeing its TMEM.
#include <cuda_runtime.h>

#include "device_types.h"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NT = 256;
constexpr int TB = KATE_TILE_BITS;  // 12 tile bits
constexpr int TS = 1 << TB;
constexpr uint32_t A_BYTES = 128 * 64 * 4;   // 32 KiB per operand (hi or lo)
constexpr uint32_t S_BYTES = TS * 8;         // 32 KiB staging tile (float2)
constexpr uint32_t OFF_A = 0;
constexpr uint32_t OFF_AL = OFF_A + A_BYTES;
constexpr uint32_t OFF_B = OFF_AL + A_BYTES;                                   // blocks' B images
constexpr uint32_t OFF_S = OFF_B + KATE_C64_MAX_BLOCKS * KATE_BLOCK_IMG_BYTES;  // two staging tiles
constexpr uint32_t OFF_MISC = OFF_S + 2 * S_BYTES;
constexpr uint32_t SMEM_BYTES = OFF_MISC + 64 + 1024;  // + alignment slack
constexpr uint32_t TMEM_COLS = 64;
constexpr long WAIT_LIMIT = 1L << 24;

// Pair-preserving swizzle of the staging tile (float2 elements): XORs bits
// 1..3 of the index with bits 4..6 and 8..10, spreading strided 8-byte
// accesses over the banks while keeping element pairs 16-byte contiguous.
__device__ __forceinline__ uint32_t sswz(uint32_t i) { return i ^ ((((i >> 4) ^ (i >> 8)) & 7u) << 1); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: 8-row groups
// 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;              // leading byte offset (16 B; unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1u << 46;              // descriptor version for sm_100
    d |= (uint64_t)2u << 61;              // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D F32, A/B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (long it = 0; it < WAIT_LIMIT; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(NT, 1)
    k_block_c64(float2* __restrict__ st, const __grid_constant__ BlockProg P, const uint8_t* __restrict__ bimg,
                int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-byte aligned operand region
    uint8_t* gbase = smem_raw + (base - raw);
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const uint32_t mbar = base + OFF_MISC;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + OFF_MISC + 8);
    int* abort_flag = reinterpret_cast<int*>(gbase + OFF_MISC + 16);

    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        *abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // Block matrices: B images into shared memory once.
    for (int b = 0; b < P.nblocks; b++) {
        const uint8_t* src = bimg + P.bimg[b];
        const uint32_t dst = base + OFF_B + b * KATE_BLOCK_IMG_BYTES;
        for (uint32_t off = t * 16; off < KATE_BLOCK_IMG_BYTES; off += NT * 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + off), "l"(src + off) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // Global offsets: tile element t + 256 j lives at dT(t) + dH(j).
    uint64_t dT = 0;
    for (int i = 0; i < 8; i++) dT |= (uint64_t)((t >> i) & 1u) << P.tphys[i];
    uint64_t dH[16];
    uint32_t oH[16];
    uint32_t pT = 0;
    for (int i = 0; i < 8; i++) pT |= ((t >> i) & 1u) << P.outsrc[i];
#pragma unroll
    for (int j = 0; j < 16; j++) {
        uint64_t g = 0;
        uint32_t o = 0;
        for (int i = 0; i < 4; i++)
            if ((j >> i) & 1) {
                g |= 1ull << P.tphys[8 + i];
                o |= 1u << P.outsrc[8 + i];
            }
        dH[j] = g;
        oH[j] = o;
    }
    auto coset_base = [&](uint64_t c) {
        uint64_t b = 0;
        for (int i = 0; i < P.ncb; i++) b |= ((c >> i) & 1ull) << P.cphys[i];
        return b;
    };
    auto prefetch = [&](uint64_t c, uint32_t sbuf) {
        const float2* src = st + coset_base(c) + dT;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t d = sbuf + sswz(t + ((uint32_t)j << 8)) * 8u;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src + dH[j]) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    const uint64_t ncos = 1ull << P.ncb;
    uint32_t phase = 0;
    if ((uint64_t)blockIdx.x < ncos) prefetch(blockIdx.x, base + OFF_S);
    int it = 0;
    for (uint64_t c = blockIdx.x; c < ncos; c += gridDim.x, it++) {
        const uint32_t sb = base + OFF_S + (uint32_t)(it & 1) * S_BYTES;
        float2* S = reinterpret_cast<float2*>(gbase + OFF_S + (it & 1) * S_BYTES);
        if (c + gridDim.x < ncos) {
            prefetch(c + gridDim.x, base + OFF_S + (uint32_t)((it + 1) & 1) * S_BYTES);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        (void)sb;

        for (int blk = 0; blk < P.nblocks; blk++) {
            // Non-block tile bits (ascending): row index bits.
            uint32_t bmask = 0;
            for (int i = 0; i < 5; i++) bmask |= 1u << P.btb[blk][i];
            // 1. A operand (hi, lo) from the staging tile. Thread t: row
            //    r = t & 127, K half h = t >> 7 (block indices 16h..16h+15).
            {
                const uint32_t r = t & 127u, h = t >> 7;
                uint32_t rbase = 0;
                for (int i = 0, q = 0; i < TB; i++)
                    if (!((bmask >> i) & 1u)) rbase |= ((r >> q++) & 1u) << i;
                const uint32_t rowoff = h * 16384u + (r >> 3) * 1024u + (r & 7u) * 128u;
#pragma unroll
                for (int cpair = 0; cpair < 8; cpair++) {
                    float v[4];
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const uint32_t b = h * 16u + (uint32_t)(2 * cpair + e);
                        uint32_t idx = rbase;
#pragma unroll
                        for (int i = 0; i < 5; i++) idx |= ((b >> i) & 1u) << P.btb[blk][i];
                        const float2 a = S[sswz(idx)];
                        v[2 * e] = a.x;
                        v[2 * e + 1] = a.y;
                    }
                    float hi[4], lo[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        hi[e] = tf32_rna(v[e]);
                        lo[e] = v[e] - hi[e];
                    }
                    const uint32_t off = rowoff + (((uint32_t)cpair ^ (r & 7u)) << 4);
                    *reinterpret_cast<float4*>(gbase + OFF_A + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
                    *reinterpret_cast<float4*>(gbase + OFF_AL + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            // 2. Tensor-core products into TMEM.
            if (t == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t bb = base + OFF_B + blk * KATE_BLOCK_IMG_BYTES;
#pragma unroll 1
                for (int s = 0; s < 8; s++) {
                    const uint32_t ka = (uint32_t)(s >> 2) * 16384u + (uint32_t)(s & 3) * 32u;
                    const uint32_t kb = (uint32_t)(s >> 2) * 8192u + (uint32_t)(s & 3) * 32u;
                    const uint64_t a_hi = sw128_desc(base + OFF_A + ka), a_lo = sw128_desc(base + OFF_AL + ka);
                    const uint64_t b_hi = sw128_desc(bb + kb), b_lo = sw128_desc(bb + 16384u + kb);
                    mma_tf32(tmem, a_hi, b_hi, s > 0 ? 1u : 0u);
                    mma_tf32(tmem, a_hi, b_lo, 1u);
                    mma_tf32(tmem, a_lo, b_hi, 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                             : "memory");
            }
            const bool ok = mbar_wait(mbar, phase);
            phase ^= 1u;
            if (!ok) *abort_flag = 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncthreads();
            if (*abort_flag) break;
            // 3. Results: warp w reads TMEM lanes 32(w&3)..+31 (rows) and
            //    columns 32(w>>2)..+31 (block indices 16(w>>2)..+15).
            {
                const uint32_t sub = warp & 3u, ch = warp >> 2;
                const uint32_t r = sub * 32u + lane;
                uint32_t d[32];
                const uint32_t taddr = tmem + ((sub * 32u) << 16) + ch * 32u;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                      "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
                      "=r"(d[15]), "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]),
                      "=r"(d[22]), "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]),
                      "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                uint32_t rbase = 0;
                for (int i = 0, q = 0; i < TB; i++)
                    if (!((bmask >> i) & 1u)) rbase |= ((r >> q++) & 1u) << i;
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    const uint32_t b = ch * 16u + (uint32_t)e;
                    uint32_t idx = rbase;
#pragma unroll
                    for (int i = 0; i < 5; i++) idx |= ((b >> i) & 1u) << P.btb[blk][i];
                    S[sswz(idx)] = make_float2(__uint_as_float(d[2 * e]), __uint_as_float(d[2 * e + 1]));
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
        }
        if (*abort_flag) break;
        // Write back with the remap permutation.
        float2* dst = st + coset_base(c) + dT;
#pragma unroll
        for (int j = 0; j < 16; j++) dst[dH[j]] = S[sswz(pT | oH[j])];
        __syncthreads();
    }
    if (*abort_flag && t == 0) atomicExch(err, 1);
    // Drain any outstanding prefetch before the CTA exits.
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

}  // namespace

int block_c64_grid(int n, int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        cudaFuncSetAttribute(k_block_c64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cached[device] = sms;
    }
    const uint64_t ncos = 1ull << (n - TB);
    return (int)(ncos < (uint64_t)cached[device] ? ncos : (uint64_t)cached[device]);
}

cudaError_t launch_block_c64(void* st, const BlockProg& prog, const void* bimg, int* err, int grid, cudaStream_t s) {
    if (prog.m != TB || prog.nblocks < 1 || prog.nblocks > KATE_C64_MAX_BLOCKS) return cudaErrorInvalidValue;
    k_block_c64<<<grid, NT, SMEM_BYTES, s>>>((float2*)st, prog, (const uint8_t*)bimg, err);
    return cudaGetLastError();
}

}  // namespace kate
