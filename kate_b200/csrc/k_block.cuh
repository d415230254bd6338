// Complex64 tensor-core blocks: the device code shared by the simulator's
// pass kernel (k_block_c64.cu) and the batch kernel's block tasks
// (k_batch.cu). A pass applies up to KATE_C64_MAX_BLOCKS dense 5-qubit blocks
// (BlockProg, device_types.h) to 4096-amplitude coset tiles staged in shared
// memory; per block:
//   1. every thread builds its part of the MMA A operand from the staging
//      tile: row r = t & 127 (the values of the 7 non-block tile bits), K
//      half h = t >> 7 (the 16 block indices 16h..16h+15, re/im interleaved),
//      as a BF16 hi part and the BF16 remainder (lo), and writes it to TMEM
//      (tcgen05.st; the A operand of tcgen05.mma may live in TMEM: lane r,
//      one 32-bit column per re/im pair);
//   2. one elected thread issues 4 K-steps x 3 products (A_hi.B_hi,
//      A_hi.B_lo, A_lo.B_hi; M = 128, N = 64, K = 16; A from TMEM, B from
//      shared memory) into one TMEM accumulator and commits to an mbarrier;
//   3. every thread reads its row's 32 results back from TMEM and writes
//      them to the staging tile at the amplitudes' tile positions.
// Then the tile is written back with the pass's remap permutation (16-byte
// stores of amplitude pairs). All waits are bounded.
//
// Accuracy: hi + lo keeps ~16 bits of each FP32 operand and the dropped
// lo.lo product is ~2^-16 relative, so one block's relative error is about
// 1e-5 per amplitude; infidelity stays orders of magnitude below 1e-6 over a
// circuit (checked against complex128 by the tests and the bench).
#pragma once

#include <cuda_runtime.h>

#include "device_types.h"

namespace kate {
namespace blk {

constexpr int NT = 256;
constexpr int TB = KATE_TILE_BITS;  // 12 tile bits
constexpr int TS = 1 << TB;
constexpr uint32_t S_BYTES = TS * 8;  // one staging tile (float2)
// TMEM columns per tile: the FP32 accumulator (N = 64), then the A
// operand's hi and lo parts (128 lanes x 64 BF16 = 32 columns each).
constexpr uint32_t TMEM_COLS = 128;
constexpr uint32_t TM_AHI = 64, TM_ALO = 96;
constexpr long WAIT_LIMIT = 1L << 24;
// Per-pass tables in shared memory: per block the swizzled tile offset of
// each block index (32 entries), then 8 swizzled copy offsets P(j << 9), 8
// write-back offsets P(oH[j]) and P(o1).
constexpr uint32_t TAB_BYTES = KATE_C64_MAX_BLOCKS * 32 * 2;
constexpr uint32_t IO_BYTES = 32 * 2;

// The pass's staging-tile swizzle (BlockProg::smask, chosen on the host):
// element e sits at e ^ sum_k parity(e & f[k]) << k. Linear over GF(2), so
// offsets of XOR-combined indices XOR.
struct Swz {
    uint32_t f0, f1, f2, f3;
    __device__ __forceinline__ uint32_t operator()(uint32_t e) const {
        return e ^ ((uint32_t)__popc(e & f0) & 1u) ^ (((uint32_t)__popc(e & f1) & 1u) << 1) ^
               (((uint32_t)__popc(e & f2) & 1u) << 2) ^ (((uint32_t)__popc(e & f3) & 1u) << 3);
    }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Two floats rounded to BF16 (nearest even) and packed: lo in bits 0..15,
// hi in bits 16..31.
__device__ __forceinline__ uint32_t bf16x2_rn(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: 8-row groups
// 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;            // leading byte offset (16 B; unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
    d |= (uint64_t)1u << 46;            // descriptor version for sm_100
    d |= (uint64_t)2u << 61;            // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D F32, A/B BF16, both K-major, N = 64, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// D (TMEM) += A (TMEM) x B (shared memory descriptor).
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// 16 consecutive TMEM columns of this warp's 32 lanes from 16 registers per thread.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
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

// Copies the pass's block operand images (nblocks x KATE_BLOCK_IMG_BYTES,
// contiguous per block, 16-byte aligned in global memory) into shared memory
// at `dst` (block b at dst + b * KATE_BLOCK_IMG_BYTES) with the bulk-copy
// engine: thread 0 announces the bytes on mbarrier `mbar` and issues one
// cp.async.bulk per image; every thread waits (bounded) for the phase
// `phase`, which it then flips. src(b) gives block b's global image.
// Returns false when the wait gave up.
template <typename Src>
__device__ __forceinline__ bool load_images(int nblocks, Src src, uint32_t dst, uint32_t mbar, uint32_t& phase) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                     "r"((uint32_t)nblocks * KATE_BLOCK_IMG_BYTES)
                     : "memory");
        for (int b = 0; b < nblocks; b++)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dst + (uint32_t)b * KATE_BLOCK_IMG_BYTES),
                "l"(src(b)), "r"((uint32_t)KATE_BLOCK_IMG_BYTES), "r"(mbar)
                : "memory");
    }
    const bool ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    return ok;
}

// TMEM allocation of one CTA, `cols` columns (a power of two, 32..512;
// warp 0 allocates; every thread reads the base after the barrier the
// caller places). `slot` is a shared-memory word.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

// Frees the CTA's TMEM; every thread calls it (it synchronises the CTA).
__device__ __forceinline__ void tmem_free(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
    }
}

// A pass's per-thread addressing, built by setup() from a BlockProg.
struct Pass {
    uint32_t rsa[KATE_C64_MAX_BLOCKS], rsr[KATE_C64_MAX_BLOCKS];  // swizzled A row / TMEM row offsets
    uint64_t dT, dH[8];  // global offsets of this thread's 8 amplitude pairs within a coset
    uint32_t cp_base, wb_base;
    bool pairs;          // amplitude pairs stay in one 16-byte staging slot
};

// Builds the pass's tables (tab, iot in shared memory) and this thread's
// addressing. The caller places a barrier before the tables are read.
__device__ __forceinline__ void setup(const BlockProg& P, uint16_t* tab, uint16_t* iot, Pass& X) {
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const Swz sswz{P.smask[0], P.smask[1], P.smask[2], P.smask[3]};
    X.pairs = P.smask[0] == 0;
#pragma unroll
    for (int blk = 0; blk < KATE_C64_MAX_BLOCKS; blk++) {
        X.rsa[blk] = X.rsr[blk] = 0;
        if (blk >= P.nblocks) continue;
        uint32_t bmask = 0;
        for (int i = 0; i < 5; i++) bmask |= 1u << P.btb[blk][i];
        const uint32_t ra = t & 127u, rr = (warp & 3u) * 32u + lane;
        uint32_t da = 0, dr = 0;
        for (int i = 0, q = 0; i < TB; i++)
            if (!((bmask >> i) & 1u)) {
                da |= ((ra >> q) & 1u) << i;
                dr |= ((rr >> q) & 1u) << i;
                q++;
            }
        X.rsa[blk] = sswz(da);
        X.rsr[blk] = sswz(dr);
        if (t < 32) {
            uint32_t idx = 0;
            for (int i = 0; i < 5; i++) idx |= ((t >> i) & 1u) << P.btb[blk][i];
            tab[blk * 32 + t] = (uint16_t)sswz(idx);
        }
    }
    // Copy j of thread t moves the amplitude pair e, e + 1 with e = 2t + 512 j
    // (tile bit 0 is physical bit 0): global offset dT + dH[j]; on write-back
    // the pair reads the tile at pT | oH[j] and (pT | oH[j]) | o1.
    uint64_t dT = 0;
    uint32_t pT = 0;
    for (int i = 0; i < 8; i++) {
        dT |= (uint64_t)((t >> i) & 1u) << P.tphys[i + 1];
        pT |= ((t >> i) & 1u) << P.outsrc[i + 1];
    }
    X.dT = dT;
    uint32_t oH[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        uint64_t g = 0;
        uint32_t o = 0;
        for (int i = 0; i < 3; i++)
            if ((j >> i) & 1) {
                g |= 1ull << P.tphys[9 + i];
                o |= 1u << P.outsrc[9 + i];
            }
        X.dH[j] = g;
        oH[j] = o;
    }
    const uint32_t o1 = 1u << P.outsrc[0];
    if (t < 8) {
        iot[t] = (uint16_t)sswz((uint32_t)t << 9);
        iot[8 + t] = (uint16_t)sswz(oH[t]);
    } else if (t == 8) {
        iot[16] = (uint16_t)sswz(o1);
    }
    X.cp_base = sswz(2u * t);  // copy-in: element 2t + 512 j at cp_base ^ iot[j]
    X.wb_base = sswz(pT);      // write-back: output pair j reads wb_base ^ iot[8 + j]
}

__device__ __forceinline__ uint64_t coset_base(const BlockProg& P, uint64_t c) {
    uint64_t b = 0;
    for (int i = 0; i < P.ncb; i++) b |= ((c >> i) & 1ull) << P.cphys[i];
    return b;
}

// Issues the copy of the tile at global base `cb` into the staging tile at
// shared address `sb` (no commit: the caller commits the group). Pairs go
// through L2 only (cp.async.cg). L2ONLY: the state may have been written by
// other SMs earlier in the same launch, so an unpaired swizzle's 8-byte
// copies (which cp.async can only route through L1) become L2 loads and
// shared stores, visible after the caller's barrier.
template <bool L2ONLY>
__device__ __forceinline__ void load_tile(const float2* st, uint64_t cb, uint32_t sb, const Pass& X,
                                          const uint16_t* iot) {
    const float2* src = st + cb + X.dT;
    if (X.pairs) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t d = sb + (X.cp_base ^ iot[j]) * 8u;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + X.dH[j]) : "memory");
        }
    } else if (L2ONLY) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t e0 = X.cp_base ^ iot[j];
            const float4 v = __ldcg(reinterpret_cast<const float4*>(src + X.dH[j]));
            asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(sb + e0 * 8u), "f"(v.x), "f"(v.y) : "memory");
            asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(sb + (e0 ^ 1u) * 8u), "f"(v.z), "f"(v.w)
                         : "memory");
        }
    } else {
        // The pair's two amplitudes land in different 8-byte slots.
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t e0 = X.cp_base ^ iot[j];
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sb + e0 * 8u), "l"(src + X.dH[j])
                         : "memory");
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sb + (e0 ^ 1u) * 8u),
                         "l"(src + X.dH[j] + 1)
                         : "memory");
        }
    }
}

// Fills the staging tile with the tile of |0...0>: zeros, and 1 at element
// 0 when `one` (coset 0; element 0 sits at staging offset 0 since the
// swizzle is linear).
__device__ __forceinline__ void zero_tile(float2* S, bool one) {
    float4* s4 = reinterpret_cast<float4*>(S);
    for (uint32_t i = threadIdx.x; i < (uint32_t)TS / 2; i += NT) s4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    if (one && threadIdx.x == 0) S[0] = make_float2(1.f, 0.f);
}

// Applies the pass's blocks to NTL staging tiles S[0..NTL) in lock-step
// (each copy complete and visible to every thread). Tile i uses the 128 TMEM
// columns from tmem + 128 i (accumulator, then the A parts). Per block: the
// A operands of every tile, one barrier, one batch of products for all
// tiles behind one mbarrier, the read-backs, one barrier; two tiles halve the
// barriers and product round trips per tile. B images at shared address
// bimg (block b at bimg + b * KATE_BLOCK_IMG_BYTES, 1024-byte aligned).
// Returns false when a product wait gave up (after every thread has left
// the block loop).
template <int NTL>
__device__ __forceinline__ bool apply_blocks(const BlockProg& P, const Pass& X, const uint16_t* tab,
                                             float2* const (&S)[NTL], uint32_t bimg, uint32_t tmem, uint32_t mbar,
                                             uint32_t& phase, int* abort_flag) {
    const uint32_t t = threadIdx.x, warp = t >> 5;
    for (int blk = 0; blk < P.nblocks; blk++) {
        const uint16_t* tb = tab + blk * 32;
        const uint32_t ra_sw = blk == 0 ? X.rsa[0] : X.rsa[KATE_C64_MAX_BLOCKS - 1];
        const uint32_t rr_sw = blk == 0 ? X.rsr[0] : X.rsr[KATE_C64_MAX_BLOCKS - 1];
        const bool wide = P.btb[blk][0] == 0 && X.pairs;  // block index bits 0 = tile bit 0: 16-byte pairs
        // 1. A operands (hi, lo) from the staging tiles into TMEM. Thread t:
        //    row r = t & 127 (TMEM lane 32 (warp & 3) + lane), K half
        //    h = t >> 7 (block indices 16h..16h+15: TMEM columns 16h..16h+15
        //    of the A parts, one re/im pair per column).
#pragma unroll
        for (int ti = 0; ti < NTL; ti++) {
            const float2* St = S[ti];
            const uint32_t h = t >> 7;
            uint32_t hw[16], lw[16];
            auto split = [&](int e, float2 a) {
                const uint32_t hp = bf16x2_rn(a.x, a.y);
                const float hre = __uint_as_float(hp << 16), him = __uint_as_float(hp & 0xffff0000u);
                hw[e] = hp;
                lw[e] = bf16x2_rn(a.x - hre, a.y - him);
            };
            if (wide) {
#pragma unroll
                for (int e = 0; e < 16; e += 2) {
                    const float4 v = *reinterpret_cast<const float4*>(&St[ra_sw ^ tb[h * 16u + (uint32_t)e]]);
                    split(e, make_float2(v.x, v.y));
                    split(e + 1, make_float2(v.z, v.w));
                }
            } else {
#pragma unroll
                for (int e = 0; e < 16; e++) split(e, St[ra_sw ^ tb[h * 16u + (uint32_t)e]]);
            }
            const uint32_t lane_base = tmem + (uint32_t)ti * 128u + (((warp & 3u) * 32u) << 16) + h * 16u;
            tmem_st16(lane_base + TM_AHI, hw);
            tmem_st16(lane_base + TM_ALO, lw);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // 2. Tensor-core products into TMEM, every tile behind one commit.
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t bb = bimg + (uint32_t)blk * KATE_BLOCK_IMG_BYTES;
#pragma unroll
            for (int ti = 0; ti < NTL; ti++) {
                const uint32_t tm = tmem + (uint32_t)ti * 128u;
#pragma unroll 1
                for (int s = 0; s < 4; s++) {
                    const uint32_t k = (uint32_t)s * 32u;  // K = 16 BF16 = 32 bytes per step (B)
                    const uint32_t kc = (uint32_t)s * 8u;  // K = 16 BF16 = 8 TMEM columns per step (A)
                    const uint64_t b_hi = sw128_desc(bb + k), b_lo = sw128_desc(bb + KATE_BLOCK_IMG_BYTES / 2 + k);
                    mma_bf16_ts(tm, tm + TM_AHI + kc, b_hi, s > 0 ? 1u : 0u);
                    mma_bf16_ts(tm, tm + TM_AHI + kc, b_lo, 1u);
                    mma_bf16_ts(tm, tm + TM_ALO + kc, b_hi, 1u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                         : "memory");
        }
        // Every thread waits for the products itself (try_wait suspends the
        // waiting thread), so no CTA barrier sits between the products and
        // the read-back. A wait that gives up raises the flag; the read-back
        // still runs (its values are then unused) so that every thread
        // reaches the barrier below, after which all see the flag.
        if (!mbar_wait(mbar, phase)) *abort_flag = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // 3. Results: warp w reads TMEM lanes 32(w&3)..+31 (rows) and columns
        //    32(w>>2)..+31 (block indices 16(w>>2)..+15) of each tile.
#pragma unroll
        for (int ti = 0; ti < NTL; ti++) {
            float2* St = S[ti];
            const uint32_t sub = warp & 3u, ch = warp >> 2;
            uint32_t d[32];
            const uint32_t taddr = tmem + (uint32_t)ti * 128u + ((sub * 32u) << 16) + ch * 32u;
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
            if (wide) {
#pragma unroll
                for (int e = 0; e < 16; e += 2)
                    *reinterpret_cast<float4*>(&St[rr_sw ^ tb[ch * 16u + (uint32_t)e]]) =
                        make_float4(__uint_as_float(d[2 * e]), __uint_as_float(d[2 * e + 1]),
                                    __uint_as_float(d[2 * e + 2]), __uint_as_float(d[2 * e + 3]));
            } else {
#pragma unroll
                for (int e = 0; e < 16; e++)
                    St[rr_sw ^ tb[ch * 16u + (uint32_t)e]] =
                        make_float2(__uint_as_float(d[2 * e]), __uint_as_float(d[2 * e + 1]));
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (*abort_flag) return false;
    }
    return true;
}

// Writes the staging tile back with the remap permutation, an amplitude pair
// per store. st_cg: stores that bypass L1 (the state is read by other SMs
// later in the same launch).
template <bool CG>
__device__ __forceinline__ void store_tile(const BlockProg& P, const Pass& X, const uint16_t* iot, float2* st,
                                           uint64_t cb, const float2* S) {
    float2* dst = st + cb + X.dT;
    const uint32_t po1 = iot[16];
    auto put = [&](float2* p, float4 v) {
        if (CG) __stcg(reinterpret_cast<float4*>(p), v);
        else *reinterpret_cast<float4*>(p) = v;
    };
    if (P.outsrc[0] == 0 && X.pairs) {
        // Output bit 0 keeps input bit 0: the pair is one 16-byte slot.
#pragma unroll
        for (int j = 0; j < 8; j++) put(dst + X.dH[j], *reinterpret_cast<const float4*>(&S[X.wb_base ^ iot[8 + j]]));
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t e0 = X.wb_base ^ iot[8 + j];
            const float2 v0 = S[e0], v1 = S[e0 ^ po1];
            put(dst + X.dH[j], make_float4(v0.x, v0.y, v1.x, v1.y));
        }
    }
}

}  // namespace blk
}  // namespace kate
