// Register-staged complex128 tile kernel: one group pass over the state.
//
// Each CTA (256 threads) owns one 4096-amplitude coset tile at a time, in a
// grid-stride loop over cosets:
//   1. the tile is copied global -> shared with 16-byte cp.async (each warp
//      instruction reads runs of 2^c contiguous amplitudes, c >= 4); the
//      copy of the next coset is issued before the current one is processed
//      (two 64 KiB buffers, one CTA per SM), so HBM reads overlap compute;
//   2. the pass program runs: a register stage loads 16 amplitudes per
//      thread from shared memory, applies its ops in registers (2x2, H,
//      controlled X, controlled phase, one-qubit diagonal), and stores them
//      back at the next stage boundary; shared-memory ops (dense blocks,
//      multi-qubit diagonals) run between stages;
//   3. the tile is written back to global with its tile bits permuted (the
//      qubit remap), again in contiguous runs.
// The program is a __grid_constant__ kernel parameter, so every thread reads
// the same op from the constant bank. This replaces the reference's
// per-group kernel (HIPcode/simulator.hpp:143-218) and its per-gate device
// switch (HIPcode/GPUGate.hpp:21-203).
#include "k_common.cuh"
#include "k_ops.cuh"
#include "launch.hpp"

namespace kate {

namespace {

constexpr int NT = 256;
constexpr int TB = KATE_TILE_BITS;
constexpr int TS = 1 << TB;
static_assert(NT * 16 == TS, "16 amplitudes per thread");

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ double2 mat(const PassProg& P, uint32_t i) {
    return make_double2(P.mats[i][0], P.mats[i][1]);
}

// r = u0 * x + u1 * y (complex), 8 FP64 ops.
__device__ __forceinline__ double2 row2(double2 u0, double2 u1, double2 x, double2 y) {
    double2 r;
    r.x = u0.x * x.x;
    r.x = fma(-u0.y, x.y, r.x);
    r.x = fma(u1.x, y.x, r.x);
    r.x = fma(-u1.y, y.y, r.x);
    r.y = u0.x * x.y;
    r.y = fma(u0.y, x.x, r.y);
    r.y = fma(u1.x, y.y, r.y);
    r.y = fma(u1.y, y.x, r.y);
    return r;
}

template <int B>
__device__ __forceinline__ void reg_u(double2 (&a)[16], double2 u00, double2 u01, double2 u10, double2 u11) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const double2 x = a[j], y = a[k];
        a[j] = row2(u00, u01, x, y);
        a[k] = row2(u10, u11, x, y);
    }
}

template <int B>
__device__ __forceinline__ void reg_h(double2 (&a)[16]) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const double2 x = a[j], y = a[k];
        const double2 n0 = make_double2((x.x + y.x) * KATE_SQRT2INV, (x.y + y.y) * KATE_SQRT2INV);
        a[j] = n0;
        a[k] = make_double2(n0.x - y.x * KATE_SQRT2, n0.y - y.y * KATE_SQRT2);
    }
}

template <int B>
__device__ __forceinline__ void reg_x(double2 (&a)[16], uint32_t creg) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        if (((uint32_t)j & creg) != creg) continue;
        const int k = j | (1 << B);
        const double2 x = a[j];
        a[j] = a[k];
        a[k] = x;
    }
}

// Real 2x2 [[a, b], [c, d]]: 4 FP64 ops per amplitude.
template <int B>
__device__ __forceinline__ void reg_ur(double2 (&a)[16], double u00, double u01, double u10, double u11) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const double2 x = a[j], y = a[k];
        a[j] = make_double2(fma(u01, y.x, u00 * x.x), fma(u01, y.y, u00 * x.y));
        a[k] = make_double2(fma(u11, y.x, u10 * x.x), fma(u11, y.y, u10 * x.y));
    }
}

// [[a, ib], [ic, d]] with a, b, c, d real (RX-like): 4 FP64 ops per amplitude.
template <int B>
__device__ __forceinline__ void reg_ux(double2 (&a)[16], double u00, double u01i, double u10i, double u11) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const double2 x = a[j], y = a[k];
        a[j] = make_double2(fma(-u01i, y.y, u00 * x.x), fma(u01i, y.x, u00 * x.y));
        a[k] = make_double2(fma(-u10i, x.y, u11 * y.x), fma(u10i, x.x, u11 * y.y));
    }
}

// Controlled NOT with a per-thread condition: selects, no branches.
template <int B>
__device__ __forceinline__ void reg_xs(double2 (&a)[16], uint32_t creg, bool go) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        if (((uint32_t)j & creg) != creg) continue;
        const int k = j | (1 << B);
        const double2 x = a[j], y = a[k];
        a[j] = make_double2(go ? y.x : x.x, go ? y.y : x.y);
        a[k] = make_double2(go ? x.x : y.x, go ? x.y : y.y);
    }
}

// The swizzle is linear over GF(2): swz(a | b) = swz(a) ^ swz(b) for
// disjoint a, b. A stage's shared-memory byte offset of register j is
// therefore s0 ^ W(j), W(j) the XOR of w_i over the set bits i of j.
__device__ __forceinline__ uint32_t reg_off(int j, uint32_t s0, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    return s0 ^ ((j & 1) ? w0 : 0u) ^ ((j & 2) ? w1 : 0u) ^ ((j & 4) ? w2 : 0u) ^ ((j & 8) ? w3 : 0u);
}

// Compile-time swizzle of (j << 8), j < 16.
__host__ __device__ constexpr uint32_t swz_hi(int j) {
    return ((uint32_t)j << 8) ^ ((((uint32_t)j << 5) ^ ((uint32_t)j << 2) ^ ((uint32_t)j >> 1)) & 7u);
}

__device__ __forceinline__ double2 lds(uint32_t addr) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ void sts(uint32_t addr, double2 v) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
}

// Shared-memory layout of one CTA: NBUF tiles of 4096 amplitudes (64 KiB
// each), then the per-CTA tables.
struct TileTables {
    SOp ops[KATE_MAX_SOPS];        // the pass program, copied from the kernel parameter
    double2 mats[KATE_MAX_MATS];
    uint64_t cb[3][256];   // coset base = cb[0][c & 255] | cb[1][(c >> 8) & 255] | cb[2][c >> 16]
    uint64_t goff[16];     // global offset of tile element t + 256 j is dT[t] + goff[j]
    uint64_t dT[NT];       // per-thread constants, kept here rather than in registers
    uint32_t tls[NT];      // swizzled byte offset of tile element t
    uint32_t pTs[NT];      // swizzled byte offset of the source of output element t
    uint32_t osw[16];      // swizzled byte offset of the source of output element t + 256 j: pTs(t) ^ osw[j]
    uint16_t stab[KATE_MAX_STAGES][44];
};

template <int NBUF>
constexpr size_t tile_smem_bytes() {
    return (size_t)NBUF * TS * sizeof(double2) + sizeof(TileTables);
}

// SM: whether the program has shared-memory ops (the variant without them
// has no call in its loop, so nothing is spilled around it). NBUF = 2: one
// CTA per SM, the next coset prefetched while the current one is processed;
// NBUF = 1: two CTAs per SM overlap each other's load and compute phases.
template <bool SM, int NBUF>
__global__ void __launch_bounds__(NT, 3 - NBUF)
    k_tile_c128(double2* __restrict__ st, const __grid_constant__ PassProg P, const DevOp* __restrict__ sops,
                const double2* __restrict__ pool) {
    extern __shared__ __align__(16) double2 bufs[];
    TileTables& T = *reinterpret_cast<TileTables*>(bufs + NBUF * TS);
    const uint32_t t = threadIdx.x;
    {
        // Coset-base tables: deposit of the coset index bits into the
        // non-tile physical bits, 8 index bits per table.
        for (int part = 0; part < 3; part++) {
            uint64_t b = 0;
            for (int i = 0; i < 8; i++) {
                const int bit = part * 8 + i;
                if (bit < P.ncb && ((t >> i) & 1u)) b |= 1ull << P.cphys[bit];
            }
            T.cb[part][t] = b;
        }
        if (t < 16) {
            uint64_t g = 0;
            uint32_t o = 0;
            for (int i = 0; i < 4; i++)
                if ((t >> i) & 1u) {
                    g |= 1ull << P.tphys[8 + i];
                    o |= 1u << P.outsrc[8 + i];
                }
            T.goff[t] = g;
            T.osw[t] = ops::swz(o) << 4;
        }
        for (int i = t; i < P.nstages * 44; i += NT) (&T.stab[0][0])[i] = (&P.stab[0][0])[i];
        for (int i = t; i < P.nops; i += NT) T.ops[i] = P.ops[i];
        for (int i = t; i < P.nmats; i += NT) T.mats[i] = make_double2(P.mats[i][0], P.mats[i][1]);
    }
    {
        uint64_t dT = 0;
        uint32_t pT = 0;
        for (int i = 0; i < 8; i++) {
            dT |= (uint64_t)((t >> i) & 1u) << P.tphys[i];
            pT |= ((t >> i) & 1u) << P.outsrc[i];
        }
        T.dT[t] = dT;
        T.pTs[t] = ops::swz(pT) << 4;
        T.tls[t] = ops::swz(t) << 4;
    }
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(bufs);
    __syncthreads();
    const uint32_t ncos = 1u << P.ncb;
    auto coset_base = [&](uint32_t c) { return T.cb[0][c & 255u] | T.cb[1][(c >> 8) & 255u] | T.cb[2][c >> 16]; };
    auto load = [&](uint32_t c, uint32_t buf) {
        const double2* src = st + (coset_base(c) + T.dT[t]);
        const uint32_t tls = T.tls[t];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t d = buf + (tls ^ (swz_hi(j) << 4));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + T.goff[j]) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    if (NBUF == 2 && blockIdx.x < ncos) load(blockIdx.x, sbase);
    int it = 0;
    for (uint32_t c = blockIdx.x; c < ncos; c += gridDim.x, it++) {
        const uint32_t tb = sbase + (uint32_t)((NBUF == 2 ? (it & 1) : 0) * TS * sizeof(double2));
        double2* tile = bufs + (NBUF == 2 ? (it & 1) : 0) * TS;
        if (NBUF == 2) {
            // Prefetch the next coset into the other buffer, then wait for this one.
            if (c + gridDim.x < ncos) {
                load(c + gridDim.x, sbase + (uint32_t)(((it + 1) & 1) * TS * sizeof(double2)));
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
        } else {
            load(c, sbase);
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();

        double2 a[16];
        bool open = false;
        uint32_t s0s = 0;   // store offset base of the open stage (flipped by SOP_XF)
        uint32_t lflip = 0; // load offset flips for the next stage (SOP_XL)
        int si = 0;         // open stage's table
        // Stores the open stage's registers through its store basis.
        auto store_regs = [&]() {
            const uint16_t* tab = T.stab[si];
            const uint32_t v0 = tab[36], v1 = tab[37], v2 = tab[38], v3 = tab[39];
#pragma unroll
            for (int j = 0; j < 16; j++) sts(tb + reg_off(j, s0s, v0, v1, v2, v3), a[j]);
        };
        for (int k = 0; k < P.nops; k++) {
            const SOp op = T.ops[k];
            switch (op.kind) {
            case SOP_STAGE: {
                if (open) store_regs();
                __syncthreads();
                si = op.idx;
                const uint16_t* tab = T.stab[si];
                const uint32_t s0 = (uint32_t)tab[t & 15u] ^ (uint32_t)tab[16 + (t >> 4)];
                const uint32_t w0 = tab[32], w1 = tab[33], w2 = tab[34], w3 = tab[35];
                const uint32_t sl = s0 ^ lflip;
#pragma unroll
                for (int j = 0; j < 16; j++) a[j] = lds(tb + reg_off(j, sl, w0, w1, w2, w3));
                s0s = s0;
                lflip = 0;
                open = true;
                break;
            }
            case SOP_XF: {
                if ((t & op.cthr) == op.cthr && (op.ccos == 0 || (coset_base(c) & op.ccos) == op.ccos)) s0s ^= op.idx;
                break;
            }
            case SOP_XL: {
                if ((t & op.cthr) == op.cthr && (op.ccos == 0 || (coset_base(c) & op.ccos) == op.ccos)) lflip ^= op.idx;
                break;
            }
            case SOP_SMEM: {
                if (!SM) break;
                if (open) {
                    store_regs();
                    open = false;
                }
                // The registers are dead until the next stage loads them.
#pragma unroll
                for (int j = 0; j < 16; j++) a[j] = make_double2(0.0, 0.0);
                __syncthreads();
                const DevOp d = sops[P.sop0 + op.idx];
                ops::apply_op(tile, TB, coset_base(c), d, pool, (int)t, NT);
                __syncthreads();
                break;
            }
            case SOP_U: {
                const double2 u00 = T.mats[op.idx], u01 = T.mats[op.idx + 1], u10 = T.mats[op.idx + 2],
                              u11 = T.mats[op.idx + 3];
                switch (op.a) {
                case 0: reg_u<0>(a, u00, u01, u10, u11); break;
                case 1: reg_u<1>(a, u00, u01, u10, u11); break;
                case 2: reg_u<2>(a, u00, u01, u10, u11); break;
                default: reg_u<3>(a, u00, u01, u10, u11); break;
                }
                break;
            }
            case SOP_UR: {
                const double u00 = T.mats[op.idx].x, u01 = T.mats[op.idx + 1].x, u10 = T.mats[op.idx + 2].x,
                             u11 = T.mats[op.idx + 3].x;
                switch (op.a) {
                case 0: reg_ur<0>(a, u00, u01, u10, u11); break;
                case 1: reg_ur<1>(a, u00, u01, u10, u11); break;
                case 2: reg_ur<2>(a, u00, u01, u10, u11); break;
                default: reg_ur<3>(a, u00, u01, u10, u11); break;
                }
                break;
            }
            case SOP_UX: {
                const double u00 = T.mats[op.idx].x, u01 = T.mats[op.idx + 1].y, u10 = T.mats[op.idx + 2].y,
                             u11 = T.mats[op.idx + 3].x;
                switch (op.a) {
                case 0: reg_ux<0>(a, u00, u01, u10, u11); break;
                case 1: reg_ux<1>(a, u00, u01, u10, u11); break;
                case 2: reg_ux<2>(a, u00, u01, u10, u11); break;
                default: reg_ux<3>(a, u00, u01, u10, u11); break;
                }
                break;
            }
            case SOP_H: {
                switch (op.a) {
                case 0: reg_h<0>(a); break;
                case 1: reg_h<1>(a); break;
                case 2: reg_h<2>(a); break;
                default: reg_h<3>(a); break;
                }
                break;
            }
            case SOP_X: {
                const bool go = (t & op.cthr) == op.cthr && (op.ccos == 0 || (coset_base(c) & op.ccos) == op.ccos);
                if (op.cthr == 0) {  // warp-uniform condition: branch
                    if (!go) break;
                    switch (op.a) {
                    case 0: reg_x<0>(a, op.creg); break;
                    case 1: reg_x<1>(a, op.creg); break;
                    case 2: reg_x<2>(a, op.creg); break;
                    default: reg_x<3>(a, op.creg); break;
                    }
                } else {
                    switch (op.a) {
                    case 0: reg_xs<0>(a, op.creg, go); break;
                    case 1: reg_xs<1>(a, op.creg, go); break;
                    case 2: reg_xs<2>(a, op.creg, go); break;
                    default: reg_xs<3>(a, op.creg, go); break;
                    }
                }
                break;
            }
            case SOP_PH: {
                if ((t & op.cthr) != op.cthr || (op.ccos != 0 && (coset_base(c) & op.ccos) != op.ccos)) break;
                const double2 ph = T.mats[op.idx];
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (((uint32_t)j & op.creg) == op.creg) a[j] = cmul(a[j], ph);
                break;
            }
            case SOP_D1: {
                const double2 d0 = T.mats[op.idx], d1 = T.mats[op.idx + 1];
                const bool b =
                    op.src == SRC_THR ? ((t >> op.a) & 1u) : (uint32_t)((coset_base(c) >> op.a) & 1ull);
                const double2 d = b ? d1 : d0;
#pragma unroll
                for (int j = 0; j < 16; j++) a[j] = cmul(a[j], d);
                break;
            }
            case SOP_DR: {
#pragma unroll
                for (int j = 0; j < 16; j++) a[j] = cmul(a[j], T.mats[op.idx + j]);
                break;
            }
            default:
                break;
            }
        }
        if (open) store_regs();
        __syncthreads();
        double2* dst = st + (coset_base(c) + T.dT[t]);
        const uint32_t pTs = T.pTs[t];
        // Four at a time: bounds the registers in flight (the op loop's
        // amplitudes are dead here, but the allocator sizes for the peak).
#pragma unroll
        for (int j0 = 0; j0 < 16; j0 += 4) {
#pragma unroll
            for (int j = j0; j < j0 + 4; j++) dst[T.goff[j]] = lds(tb + (pTs ^ T.osw[j]));
            asm volatile("" ::: "memory");
        }
        // The buffer is refilled by the next load.
        __syncthreads();
    }
}

}  // namespace

template <int NBUF>
int tile_grid_for(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        const int smem = (int)tile_smem_bytes<NBUF>();
        cudaFuncSetAttribute(k_tile_c128<true, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_tile_c128<false, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile_c128<false, NBUF>, NT, smem);
        if (occ < 1) occ = 1;
        cached[device] = sms * occ;
    }
    return cached[device];
}

int tile_pass_grid(int n, int device, int nbuf) {
    const int g = nbuf == 2 ? tile_grid_for<2>(device) : tile_grid_for<1>(device);
    const uint64_t ncos = 1ull << (n - TB);
    return (int)(ncos < (uint64_t)g ? ncos : (uint64_t)g);
}

cudaError_t launch_tile_c128(void* st, const PassProg& prog, const DevOp* sops, const void* pool, int grid, int nbuf,
                             cudaStream_t s) {
    if (prog.m != TB || prog.ncb > 22) return cudaErrorInvalidValue;
    bool sm = false;
    for (int k = 0; k < prog.nops; k++) sm |= prog.ops[k].kind == SOP_SMEM;
    double2* x = (double2*)st;
    const double2* pl = (const double2*)pool;
    if (nbuf == 2) {
        const size_t smem = tile_smem_bytes<2>();
        if (sm) k_tile_c128<true, 2><<<grid, NT, smem, s>>>(x, prog, sops, pl);
        else k_tile_c128<false, 2><<<grid, NT, smem, s>>>(x, prog, sops, pl);
    } else {
        const size_t smem = tile_smem_bytes<1>();
        if (sm) k_tile_c128<true, 1><<<grid, NT, smem, s>>>(x, prog, sops, pl);
        else k_tile_c128<false, 1><<<grid, NT, smem, s>>>(x, prog, sops, pl);
    }
    return cudaGetLastError();
}

}  // namespace kate
