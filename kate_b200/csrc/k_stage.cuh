// Register-staged pass programs on one 4096-amplitude coset tile (see
// PassProg in device_types.h), for both amplitude types:
//   double2  complex128, FP64 arithmetic: 16-byte elements;
//   float2   complex64, FP32 arithmetic: 8-byte elements.
// Used by the tile kernel (k_tile.cu) and the batch kernel (k_batch.cu).
//
// Shared-memory byte offsets are tsw(e) << SH for element e: swz(e) << 4
// for complex128, swz2(e) << 3 for complex64 (see k_ops.cuh). The host
// writes stage tables and SOP_XF / SOP_XL flips as complex128 offsets,
// swz(x) << 4 for tile-index vectors x; the complex64 setup maps each to
// swz2(x) << 3 (x = swz(v >> 4), swz being its own inverse). All maps are
// linear over GF(2), so XOR combinations of table entries map alike.
#pragma once

#include "k_common.cuh"
#include "k_ops.cuh"

namespace kate {
namespace stage {
namespace {

constexpr int NT = 256;
constexpr int TB = KATE_TILE_BITS;
constexpr int TS = 1 << TB;
static_assert(NT * 16 == TS, "16 amplitudes per thread");

template <typename C2>
struct Amp;
template <>
struct Amp<double2> {
    using R = double;
    static constexpr int SH = 4;   // log2 bytes per element
    static constexpr int NCP = 16; // 16-byte copies per thread per tile
    __device__ __forceinline__ static R fm(R a, R b, R c) { return fma(a, b, c); }
    __device__ __forceinline__ static double2 mk(R x, R y) { return make_double2(x, y); }
    __device__ __forceinline__ static double2 lds(uint32_t addr) {
        double2 v;
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
        return v;
    }
    __device__ __forceinline__ static void sts(uint32_t addr, double2 v) {
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
    }
};
template <>
struct Amp<float2> {
    using R = float;
    static constexpr int SH = 3;
    static constexpr int NCP = 8;  // each 16-byte copy moves an adjacent pair of amplitudes
    __device__ __forceinline__ static R fm(R a, R b, R c) { return fmaf(a, b, c); }
    // Packed FP32 (sm_100): s * v, s * v + w, and i * v.
    __device__ __forceinline__ static float2 mul_s(R s, float2 v) { return __fmul2_rn(make_float2(s, s), v); }
    __device__ __forceinline__ static float2 fma_s(R s, float2 v, float2 w) { return __ffma2_rn(make_float2(s, s), v, w); }
    __device__ __forceinline__ static float2 rot(float2 v) { return make_float2(-v.y, v.x); }
    __device__ __forceinline__ static float2 mk(R x, R y) { return make_float2(x, y); }
    __device__ __forceinline__ static float2 lds(uint32_t addr) {
        float2 v;
        asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
        return v;
    }
    __device__ __forceinline__ static void sts(uint32_t addr, float2 v) {
        asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
    }
};

// r = u0 * x + u1 * y (complex): 8 FMA-class ops (complex64: 4 packed ops
// on x, y and their i-rotations).
__device__ __forceinline__ float2 row2(float2 u0, float2 u1, float2 x, float2 y) {
    using A = Amp<float2>;
    return A::fma_s(u1.y, A::rot(y), A::fma_s(u1.x, y, A::fma_s(u0.y, A::rot(x), A::mul_s(u0.x, x))));
}
template <typename C2>
__device__ __forceinline__ C2 row2(C2 u0, C2 u1, C2 x, C2 y) {
    using A = Amp<C2>;
    C2 r;
    r.x = u0.x * x.x;
    r.x = A::fm(-u0.y, x.y, r.x);
    r.x = A::fm(u1.x, y.x, r.x);
    r.x = A::fm(-u1.y, y.y, r.x);
    r.y = u0.x * x.y;
    r.y = A::fm(u0.y, x.x, r.y);
    r.y = A::fm(u1.x, y.y, r.y);
    r.y = A::fm(u1.y, y.x, r.y);
    return r;
}

template <int B, typename C2>
__device__ __forceinline__ void reg_u(C2 (&a)[16], C2 u00, C2 u01, C2 u10, C2 u11) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        a[j] = row2(u00, u01, x, y);
        a[k] = row2(u10, u11, x, y);
    }
}

// Dense two-qubit gate on register bits A (matrix index bit 0) and B (bit
// 1), matrix M (4x4 row-major, complex128 only).
template <int A, int B>
__device__ __forceinline__ void reg_u2(double2 (&a)[16], const double2* M) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if (((j >> A) & 1) || ((j >> B) & 1)) continue;
        const int r1 = j | (1 << A), r2 = j | (1 << B), r3 = j | (1 << A) | (1 << B);
        const double2 x0 = a[j], x1 = a[r1], x2 = a[r2], x3 = a[r3];
        double2 y[4];
#pragma unroll
        for (int row = 0; row < 4; row++) {
            y[row] = cmul(M[4 * row], x0);
            cfma(y[row], M[4 * row + 1], x1);
            cfma(y[row], M[4 * row + 2], x2);
            cfma(y[row], M[4 * row + 3], x3);
        }
        a[j] = y[0];
        a[r1] = y[1];
        a[r2] = y[2];
        a[r3] = y[3];
    }
}

template <int B, typename C2>
__device__ __forceinline__ void reg_h(C2 (&a)[16]) {
    using R = typename Amp<C2>::R;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        if constexpr (sizeof(C2) == 8) {
            const float2 n0 = Amp<float2>::mul_s((R)KATE_SQRT2INV, __fadd2_rn(x, y));
            a[j] = n0;
            a[k] = Amp<float2>::fma_s(-(R)KATE_SQRT2, y, n0);
        } else {
            const C2 n0 = Amp<C2>::mk((x.x + y.x) * (R)KATE_SQRT2INV, (x.y + y.y) * (R)KATE_SQRT2INV);
            a[j] = n0;
            a[k] = Amp<C2>::mk(n0.x - y.x * (R)KATE_SQRT2, n0.y - y.y * (R)KATE_SQRT2);
        }
    }
}

template <int B, typename C2>
__device__ __forceinline__ void reg_x(C2 (&a)[16], uint32_t creg) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        if (((uint32_t)j & creg) != creg) continue;
        const int k = j | (1 << B);
        const C2 x = a[j];
        a[j] = a[k];
        a[k] = x;
    }
}

// Real 2x2 [[a, b], [c, d]]: 4 FMA-class ops per amplitude.
template <int B, typename C2, typename R>
__device__ __forceinline__ void reg_ur(C2 (&a)[16], R u00, R u01, R u10, R u11) {
    using A = Amp<C2>;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        if constexpr (sizeof(C2) == 8) {
            a[j] = Amp<float2>::fma_s(u01, y, Amp<float2>::mul_s(u00, x));
            a[k] = Amp<float2>::fma_s(u11, y, Amp<float2>::mul_s(u10, x));
        } else {
            a[j] = A::mk(A::fm(u01, y.x, u00 * x.x), A::fm(u01, y.y, u00 * x.y));
            a[k] = A::mk(A::fm(u11, y.x, u10 * x.x), A::fm(u11, y.y, u10 * x.y));
        }
    }
}

// [[a, ib], [ic, d]] with a, b, c, d real (RX-like): 4 FMA-class ops per amplitude.
template <int B, typename C2, typename R>
__device__ __forceinline__ void reg_ux(C2 (&a)[16], R u00, R u01i, R u10i, R u11) {
    using A = Amp<C2>;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        if constexpr (sizeof(C2) == 8) {
            using F = Amp<float2>;
            a[j] = F::fma_s(u01i, F::rot(y), F::mul_s(u00, x));
            a[k] = F::fma_s(u10i, F::rot(x), F::mul_s(u11, y));
        } else {
            a[j] = A::mk(A::fm(-u01i, y.y, u00 * x.x), A::fm(u01i, y.x, u00 * x.y));
            a[k] = A::mk(A::fm(-u10i, x.y, u11 * y.x), A::fm(u10i, x.x, u11 * y.y));
        }
    }
}

// Rotations with their common factor taken out (SOP_URA/URB/UXA/UXB): one
// FMA-class op per real component (one packed FMA per complex64 amplitude).
//   F = 0 (URA): x0 + t0 x1,    t1 x0 + x1
//   F = 1 (URB): t0 x0 + x1,    t1 x1 - x0
//   F = 2 (UXA): x0 + i t0 x1,  x1 + i t1 x0
//   F = 3 (UXB): x1 - i t0 x0,  x0 - i t1 x1
template <int F, int B, typename C2, typename R>
__device__ __forceinline__ void reg_rot(C2 (&a)[16], R t0, R t1) {
    using A = Amp<C2>;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        if constexpr (sizeof(C2) == 8) {
            using Fp = Amp<float2>;
            if constexpr (F == 0) {
                a[j] = Fp::fma_s(t0, y, x);
                a[k] = Fp::fma_s(t1, x, y);
            } else if constexpr (F == 1) {
                a[j] = Fp::fma_s(t0, x, y);
                a[k] = Fp::fma_s(t1, y, make_float2(-x.x, -x.y));
            } else if constexpr (F == 2) {
                a[j] = Fp::fma_s(t0, Fp::rot(y), x);
                a[k] = Fp::fma_s(t1, Fp::rot(x), y);
            } else {
                a[j] = Fp::fma_s(-t0, Fp::rot(x), y);
                a[k] = Fp::fma_s(-t1, Fp::rot(y), x);
            }
        } else {
            if constexpr (F == 0) {
                a[j] = A::mk(A::fm(t0, y.x, x.x), A::fm(t0, y.y, x.y));
                a[k] = A::mk(A::fm(t1, x.x, y.x), A::fm(t1, x.y, y.y));
            } else if constexpr (F == 1) {
                a[j] = A::mk(A::fm(t0, x.x, y.x), A::fm(t0, x.y, y.y));
                a[k] = A::mk(A::fm(t1, y.x, -x.x), A::fm(t1, y.y, -x.y));
            } else if constexpr (F == 2) {
                a[j] = A::mk(A::fm(-t0, y.y, x.x), A::fm(t0, y.x, x.y));
                a[k] = A::mk(A::fm(-t1, x.y, y.x), A::fm(t1, x.x, y.y));
            } else {
                a[j] = A::mk(A::fm(t0, x.y, y.x), A::fm(-t0, x.x, y.y));
                a[k] = A::mk(A::fm(t1, y.y, x.x), A::fm(-t1, y.x, x.y));
            }
        }
    }
}

template <int F, typename C2, typename R>
__device__ __forceinline__ void reg_rot_bit(C2 (&a)[16], int b, R t0, R t1) {
    switch (b) {
    case 0: reg_rot<F, 0>(a, t0, t1); break;
    case 1: reg_rot<F, 1>(a, t0, t1); break;
    case 2: reg_rot<F, 2>(a, t0, t1); break;
    default: reg_rot<F, 3>(a, t0, t1); break;
    }
}

// Controlled NOT with a per-thread condition: selects, no branches.
template <int B, typename C2>
__device__ __forceinline__ void reg_xs(C2 (&a)[16], uint32_t creg, bool go) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
        if ((j >> B) & 1) continue;
        if (((uint32_t)j & creg) != creg) continue;
        const int k = j | (1 << B);
        const C2 x = a[j], y = a[k];
        a[j] = Amp<C2>::mk(go ? y.x : x.x, go ? y.y : x.y);
        a[k] = Amp<C2>::mk(go ? x.x : y.x, go ? x.y : y.y);
    }
}

// The swizzle is linear over GF(2): swz(a | b) = swz(a) ^ swz(b) for
// disjoint a, b. A stage's shared-memory byte offset of register j is
// therefore s0 ^ W(j), W(j) the XOR of w_i over the set bits i of j.
__device__ __forceinline__ uint32_t reg_off(int j, uint32_t s0, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    return s0 ^ ((j & 1) ? w0 : 0u) ^ ((j & 2) ? w1 : 0u) ^ ((j & 4) ? w2 : 0u) ^ ((j & 8) ? w3 : 0u);
}

// A complex128 shared-memory offset as the same tile-index vector's offset
// in a C2 tile.
template <typename C2>
__device__ __forceinline__ uint32_t conv_off(uint32_t v) {
    if (sizeof(C2) == 16) return v;
    return ops::swz2(ops::swz(v >> 4)) << 3;
}

// Per-CTA tables of one pass program.
//   complex128: copy j of thread t moves element e = t + 256 j;
//   complex64:  copy j of thread t moves elements e, e + 1 with e = 2t + 512 j.
// Global offset of the copy: cb(c) + dT[t] + goff[j]; shared byte offset of
// its (first) element: tls[t] ^ (tsw(j << 8) << 4), resp. ^ (tsw(j << 9) << 3).
// On write-back the copy's (first) output element reads the tile at
// pTs[t] ^ osw[j] (qubit remap), and for complex64 the second one at that ^ o1.
template <typename C2>
struct TileTables {
    SOp ops[KATE_MAX_SOPS];
    C2 mats[KATE_MAX_MATS];
    uint64_t cb[3][256];   // coset base = cb[0][c & 255] | cb[1][(c >> 8) & 255] | cb[2][c >> 16]
    uint64_t goff[16];
    uint64_t dT[NT];
    uint32_t tls[NT];
    uint32_t pTs[NT];
    uint32_t osw[16];
    uint32_t o1;
    uint16_t stab[KATE_MAX_STAGES][44];
};

// Fields of a pass program the tables are built from. PassProg and the
// batch's packed programs both provide them.
struct ProgView {
    int m, ncb, nops, nmats, nstages, sop0;
    const uint8_t* tphys;
    const uint8_t* outsrc;
    const uint8_t* cphys;
    const SOp* ops;
    const double (*mats)[2];
    const uint16_t (*stab)[44];
};

__device__ __forceinline__ ProgView view(const PassProg& P) {
    ProgView v;
    v.m = P.m;
    v.ncb = P.ncb;
    v.nops = P.nops;
    v.nmats = P.nmats;
    v.nstages = P.nstages;
    v.sop0 = P.sop0;
    v.tphys = P.tphys;
    v.outsrc = P.outsrc;
    v.cphys = P.cphys;
    v.ops = P.ops;
    v.mats = P.mats;
    v.stab = P.stab;
    return v;
}

// Program part of the tables (ops, matrices, stage tables). No barrier.
template <typename C2>
__device__ __forceinline__ void setup_program(TileTables<C2>& T, const ProgView& P, uint32_t t) {
    for (int i = t; i < P.nstages * 44; i += NT) (&T.stab[0][0])[i] = (uint16_t)conv_off<C2>((&P.stab[0][0])[i]);
    for (int i = t; i < P.nops; i += NT) {
        SOp o = P.ops[i];
        if (o.kind == SOP_XF || o.kind == SOP_XL) o.idx = (uint16_t)conv_off<C2>(o.idx);
        T.ops[i] = o;
    }
    for (int i = t; i < P.nmats; i += NT) T.mats[i] = Amp<C2>::mk(P.mats[i][0], P.mats[i][1]);
}

// Global-access part of the tables (coset bases, copy offsets). No barrier.
template <typename C2>
__device__ __forceinline__ void setup_io(TileTables<C2>& T, const ProgView& P, uint32_t t) {
    constexpr int SH = Amp<C2>::SH;
    constexpr int E = SH == 4 ? 0 : 1;  // log2 elements per copy
    for (int part = 0; part < 3; part++) {
        uint64_t b = 0;
        for (int i = 0; i < 8; i++) {
            const int bit = part * 8 + i;
            if (bit < P.ncb && ((t >> i) & 1u)) b |= 1ull << P.cphys[bit];
        }
        T.cb[part][t] = b;
    }
    constexpr int HB = 8 + E;  // tile bits of the copy index j start here
    if (t < (uint32_t)(1 << (TB - HB))) {
        uint64_t g = 0;
        uint32_t o = 0;
        for (int i = 0; i < TB - HB; i++)
            if ((t >> i) & 1u) {
                g |= 1ull << P.tphys[HB + i];
                o |= 1u << P.outsrc[HB + i];
            }
        T.goff[t] = g;
        T.osw[t] = ops::tsw<C2>(o) << SH;
    }
    if (t == 0) T.o1 = ops::tsw<C2>(1u << P.outsrc[0]) << SH;
    uint64_t dT = 0;
    uint32_t pT = 0;
    for (int i = 0; i < 8; i++) {
        dT |= (uint64_t)((t >> i) & 1u) << P.tphys[i + E];
        pT |= ((t >> i) & 1u) << P.outsrc[i + E];
    }
    T.dT[t] = dT;
    T.pTs[t] = ops::tsw<C2>(pT) << SH;
    T.tls[t] = ops::tsw<C2>(t << E) << SH;
}

// Direct global I/O of the first and the last register stage (complex128):
// the first stage loads its registers straight from global memory and the
// last stores them straight back, instead of copying the tile through
// shared memory (a 16-byte store and load per amplitude each way). Usable
// when the stage's thread bits 0..3 address physical bits 0..3 (every warp
// access then still covers runs of 256 contiguous bytes) and no
// shared-memory op comes before (after) that stage.
//   ml / mh  physical offset, in amplitudes, of the low / high 6 bits of a
//            tile slot (swizzled byte offset >> 4) as the tile is read;
//   sl / sh  the same as the tile is written back (qubit remap applied);
//   lr / sr  offset of register j in the first / last stage.
// Every map is linear over GF(2), so offsets of XOR-combined slots XOR.
struct DirectIO {
    uint64_t ml[64], mh[64], sl[64], sh[64];
    uint64_t lr[16], sr[16];
    int okL, okS;
    int wl;  // every shared-memory exchange of a coset stays within a warp (see setup_direct)
};

// Physical offset of tile slot x (byte offset >> 4 in the complex128
// layout) when tile bit k sits at physical bit pos[k].
__device__ __forceinline__ uint64_t slot_phys(uint32_t x, const uint8_t* pos) {
    const uint32_t e = ops::swz(x);
    uint64_t o = 0;
    for (int k = 0; k < TB; k++)
        if ((e >> k) & 1u) o |= 1ull << pos[k];
    return o;
}

// Builds D from the program (no barrier needed before; one after).
__device__ __forceinline__ void setup_direct(DirectIO& D, const ProgView& P, uint32_t t) {
    uint8_t in[TB], out[TB];
    for (int k = 0; k < TB; k++) in[k] = P.tphys[k], out[k] = P.tphys[k];
    for (int i = 0; i < TB; i++) out[P.outsrc[i]] = P.tphys[i];
    if (t < 64) D.ml[t] = slot_phys(t, in);
    else if (t < 128) D.mh[t - 64] = slot_phys((t - 64) << 6, in);
    else if (t < 192) D.sl[t - 128] = slot_phys(t - 128, out);
    else D.sh[t - 192] = slot_phys((t - 192) << 6, out);
    int first = -1, last = -1, smem_before = 0, smem_after = 0, smem_any = 0, wide = 0;
    for (int k = 0; k < P.nops; k++) {
        const int kind = P.ops[k].kind;
        if (kind == SOP_STAGE) {
            if (first >= 0 && P.ops[k].src != 1) wide = 1;  // a boundary that needs the whole CTA
            if (first < 0) first = P.ops[k].idx;
            last = P.ops[k].idx;
            smem_after = 0;
        } else if (kind == SOP_SMEM) {
            if (first < 0) smem_before = 1;
            smem_after = 1;
            smem_any = 1;
        }
    }
    if (t < 32) {
        const bool ld = t < 16;
        const int st = ld ? first : last;
        uint32_t w = 0;
        if (st >= 0)
            for (int i = 0; i < 4; i++)
                if (((t & 15u) >> i) & 1u) w ^= P.stab[st][(ld ? 32 : 36) + i];
        (ld ? D.lr : D.sr)[t & 15u] = st >= 0 ? slot_phys(w >> 4, ld ? in : out) : 0;
    }
    if (t == 0) {
        // Lanes 0..15 of a warp differ in thread bits 0..3: their slots
        // differ by stab[st][1 << b] ^ stab[st][0].
        auto lanes_ok = [&](int st, const uint8_t* pos) {
            if (st < 0) return false;
            uint64_t acc = 0;
            for (int b = 0; b < 4; b++) {
                const uint64_t d = slot_phys((uint32_t)(P.stab[st][1 << b] ^ P.stab[st][0]) >> 4, pos);
                if (d == 0 || (d & (d - 1)) != 0) return false;
                acc |= d;
            }
            return acc == 15;
        };
        D.okL = !smem_before && lanes_ok(first, in);
        D.okS = !smem_after && lanes_ok(last, out);
        // With both ends in HBM, no shared-memory op and every boundary
        // warp-local (so every stage gives the warp index the same tile
        // bits), a coset's shared-memory slots are only touched by one warp:
        // the next coset then needs a warp barrier, not a CTA one.
        D.wl = D.okL && D.okS && !smem_any && !wide;
    }
}

template <typename C2>
__device__ __forceinline__ uint64_t coset_base(const TileTables<C2>& T, uint32_t c) {
    return T.cb[0][c & 255u] | T.cb[1][(c >> 8) & 255u] | T.cb[2][c >> 16];
}

// Issues the cp.async copies of coset c into the tile at shared address
// buf, and commits them as one group.
template <typename C2>
__device__ __forceinline__ void load_async(const TileTables<C2>& T, const C2* __restrict__ st, uint32_t c, uint32_t buf,
                                           uint32_t t) {
    constexpr int SH = Amp<C2>::SH, HB = SH == 4 ? 8 : 9;
    const C2* src = st + (coset_base(T, c) + T.dT[t]);
    const uint32_t tls = T.tls[t];
#pragma unroll
    for (int j = 0; j < Amp<C2>::NCP; j++) {
        const uint32_t d = buf + (tls ^ (ops::tsw<C2>((uint32_t)j << HB) << SH));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + T.goff[j]) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void st_pair(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st_pair_cg(float2* p, float2 a, float2 b) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(a.x, a.y, b.x, b.y));
}

// Writes the tile at shared address tb back to coset c (qubit remap
// applied). CG: stores bypass L1 (other SMs read them in the same launch).
template <typename C2, bool CG>
__device__ __forceinline__ void store_tile(const TileTables<C2>& T, C2* __restrict__ st, uint32_t c, uint32_t tb,
                                           uint32_t t) {
    using A = Amp<C2>;
    C2* dst = st + (coset_base(T, c) + T.dT[t]);
    const uint32_t pTs = T.pTs[t];
    if constexpr (A::SH == 4) {
        // Four at a time: bounds the registers in flight.
#pragma unroll
        for (int j0 = 0; j0 < 16; j0 += 4) {
#pragma unroll
            for (int j = j0; j < j0 + 4; j++) {
                const C2 v = A::lds(tb + (pTs ^ T.osw[j]));
                if (CG) __stcg(dst + T.goff[j], v);
                else dst[T.goff[j]] = v;
            }
            asm volatile("" ::: "memory");
        }
    } else {
        const uint32_t o1 = T.o1;
#pragma unroll
        for (int j0 = 0; j0 < 8; j0 += 4) {
#pragma unroll
            for (int j = j0; j < j0 + 4; j++) {
                const uint32_t o = pTs ^ T.osw[j];
                const C2 v0 = A::lds(tb + o), v1 = A::lds(tb + (o ^ o1));
                if (CG) st_pair_cg(dst + T.goff[j], v0, v1);
                else st_pair(dst + T.goff[j], v0, v1);
            }
            asm volatile("" ::: "memory");
        }
    }
}

// Barrier of the threads that run a program: the whole CTA (MODE 0), or the
// 256 consumer threads of the warp-specialised tile kernel, named barrier 1
// (MODE 1; its producer warp does not take part).
template <int MODE>
__device__ __forceinline__ void prog_bar() {
    if constexpr (MODE == 0) __syncthreads();
    else asm volatile("bar.sync 1, 256;\n" ::: "memory");
}

// Byte offset, in a tile stored in plain index order (element e at 16 e),
// of the element that a complex128 swizzled byte offset s addresses. Linear
// over GF(2) like the swizzle, so XOR combinations convert term by term.
__device__ __forceinline__ uint32_t plain_off(uint32_t s) { return ops::swz(s >> 4) << 4; }

// Runs the program in T on the tile at shared address tb (generic pointer
// tile), for coset base cbase. Ends with the last stage's registers stored;
// no trailing barrier. SM: whether the program may hold shared-memory ops.
// D (complex128 only, may be null): with D->okL the first stage loads from
// the state gst at coset base cbase, with D->okS the last stage stores there
// (DirectIO); the caller then skips the tile copy in or out.
// MODE 0: the tile arrives swizzled and barriers span the CTA. MODE 1
// (complex128, no shared-memory ops): the warp-specialised kernel; the tile
// arrives in plain index order (bulk copies cannot permute within their
// 256-byte runs), so the first stage loads through plain_off, and its
// stores, which use the swizzled order, wait behind a barrier for every
// thread's first-stage loads. D->okL is not used in this mode.
template <typename C2, bool SM, int MAXK = 5, int MODE = 0>
__device__ __forceinline__ void run_program(const TileTables<C2>& T, int nops, uint32_t tb, C2* tile, uint64_t cbase,
                                            const DevOp* __restrict__ sops, int sop0,
                                            const double2* __restrict__ pool, uint32_t t,
                                            const DirectIO* D = nullptr, C2* __restrict__ gst = nullptr) {
    static_assert(MODE == 0 || (!SM && sizeof(C2) == 16), "the warp-specialised mode runs complex128 register programs");
    using A = Amp<C2>;
    using R = typename A::R;
    C2 a[16];
    bool open = false;
    bool started = false;  // a stage has been loaded
    bool plain_open = false;  // MODE 1: the open stage was loaded from the plain-order tile
    uint32_t s0s = 0;    // store offset base of the open stage (flipped by SOP_XF)
    uint32_t lflip = 0;  // load offset flips for the next stage (SOP_XL)
    int si = 0;          // open stage's table
    auto store_regs = [&]() {
        if constexpr (MODE == 1) {
            if (plain_open) {
                prog_bar<MODE>();
                plain_open = false;
            }
        }
        const uint16_t* tab = T.stab[si];
        const uint32_t v0 = tab[36], v1 = tab[37], v2 = tab[38], v3 = tab[39];
#pragma unroll
        for (int j = 0; j < 16; j++) A::sts(tb + reg_off(j, s0s, v0, v1, v2, v3), a[j]);
    };
    for (int k = 0; k < nops; k++) {
        const SOp op = T.ops[k];
        switch (op.kind) {
        case SOP_STAGE: {
            if (open) store_regs();
            si = op.idx;
            const uint16_t* tab = T.stab[si];
            const uint32_t s0 = (uint32_t)tab[t & 15u] ^ (uint32_t)tab[16 + (t >> 4)];
            const uint32_t sl = s0 ^ lflip;
            if constexpr (MODE == 1) {
                if (!started) {
                    const uint32_t p0 = plain_off(tab[32]), p1 = plain_off(tab[33]), p2 = plain_off(tab[34]),
                                   p3 = plain_off(tab[35]), pl = plain_off(sl);
#pragma unroll
                    for (int j = 0; j < 16; j++) a[j] = A::lds(tb + reg_off(j, pl, p0, p1, p2, p3));
                    started = true;
                    plain_open = true;
                    s0s = s0;
                    lflip = 0;
                    open = true;
                    break;
                }
            }
            if constexpr (sizeof(C2) == 16 && MODE == 0) {
                if (D != nullptr && !started && D->okL) {
                    // Register and thread vectors may share tile bits (folded
                    // CNOTs), so offsets combine by XOR, never by addition.
                    const uint32_t x = sl >> 4;
                    const uint64_t base = cbase ^ D->ml[x & 63u] ^ D->mh[x >> 6];
#pragma unroll
                    for (int j = 0; j < 16; j++) a[j] = __ldcg(gst + (base ^ D->lr[j]));
                    started = true;
                    s0s = s0;
                    lflip = 0;
                    open = true;
                    break;
                }
            }
            // src = 1: both stages give the same tile bits to the warp index,
            // so each warp reloads only the slots it stored.
            if (op.src == 1) __syncwarp();
            else prog_bar<MODE>();
            const uint32_t w0 = tab[32], w1 = tab[33], w2 = tab[34], w3 = tab[35];
#pragma unroll
            for (int j = 0; j < 16; j++) a[j] = A::lds(tb + reg_off(j, sl, w0, w1, w2, w3));
            started = true;
            s0s = s0;
            lflip = 0;
            open = true;
            break;
        }
        case SOP_XF: {
            if ((t & op.cthr) == op.cthr && (op.ccos == 0 || (cbase & op.ccos) == op.ccos)) s0s ^= op.idx;
            break;
        }
        case SOP_XL: {
            if ((t & op.cthr) == op.cthr && (op.ccos == 0 || (cbase & op.ccos) == op.ccos)) lflip ^= op.idx;
            break;
        }
        case SOP_SMEM: {
            if constexpr (!SM) break;
            if (open) {
                store_regs();
                open = false;
            }
            // The registers are dead until the next stage loads them.
#pragma unroll
            for (int j = 0; j < 16; j++) a[j] = A::mk(0, 0);
            __syncthreads();
            const DevOp d = sops[sop0 + op.idx];
            ops::apply_op<C2, MAXK>(tile, TB, cbase, d, pool, (int)t, NT);
            __syncthreads();
            break;
        }
        case SOP_U: {
            const C2 u00 = T.mats[op.idx], u01 = T.mats[op.idx + 1], u10 = T.mats[op.idx + 2], u11 = T.mats[op.idx + 3];
            switch (op.a) {
            case 0: reg_u<0>(a, u00, u01, u10, u11); break;
            case 1: reg_u<1>(a, u00, u01, u10, u11); break;
            case 2: reg_u<2>(a, u00, u01, u10, u11); break;
            default: reg_u<3>(a, u00, u01, u10, u11); break;
            }
            break;
        }
        case SOP_UR: {
            const R u00 = T.mats[op.idx].x, u01 = T.mats[op.idx + 1].x, u10 = T.mats[op.idx + 2].x,
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
            const R u00 = T.mats[op.idx].x, u01 = T.mats[op.idx + 1].y, u10 = T.mats[op.idx + 2].y,
                    u11 = T.mats[op.idx + 3].x;
            switch (op.a) {
            case 0: reg_ux<0>(a, u00, u01, u10, u11); break;
            case 1: reg_ux<1>(a, u00, u01, u10, u11); break;
            case 2: reg_ux<2>(a, u00, u01, u10, u11); break;
            default: reg_ux<3>(a, u00, u01, u10, u11); break;
            }
            break;
        }
        case SOP_URA:
        case SOP_URB:
        case SOP_UXA:
        case SOP_UXB: {
            const C2 tt = T.mats[op.idx];
            const R t0 = tt.x, t1 = tt.y;
            if (op.kind == SOP_URA) reg_rot_bit<0>(a, op.a, t0, t1);
            else if (op.kind == SOP_URB) reg_rot_bit<1>(a, op.a, t0, t1);
            else if (op.kind == SOP_UXA) reg_rot_bit<2>(a, op.a, t0, t1);
            else reg_rot_bit<3>(a, op.a, t0, t1);
            break;
        }
        case SOP_U2: {
            if constexpr (sizeof(C2) == 16) {
                const double2* M = reinterpret_cast<const double2*>(&T.mats[op.idx]);
                switch (op.a * 4 + op.src) {
                case 1: reg_u2<0, 1>(a, M); break;
                case 2: reg_u2<0, 2>(a, M); break;
                case 3: reg_u2<0, 3>(a, M); break;
                case 6: reg_u2<1, 2>(a, M); break;
                case 7: reg_u2<1, 3>(a, M); break;
                default: reg_u2<2, 3>(a, M); break;
                }
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
            const bool go = (t & op.cthr) == op.cthr && (op.ccos == 0 || (cbase & op.ccos) == op.ccos);
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
            if ((t & op.cthr) != op.cthr || (op.ccos != 0 && (cbase & op.ccos) != op.ccos)) break;
            const C2 ph = T.mats[op.idx];
#pragma unroll
            for (int j = 0; j < 16; j++)
                if (((uint32_t)j & op.creg) == op.creg) a[j] = cmul_r(a[j], ph);
            break;
        }
        case SOP_D1: {
            const C2 d0 = T.mats[op.idx], d1 = T.mats[op.idx + 1];
            const bool b = op.src == SRC_THR ? ((t >> op.a) & 1u) : (uint32_t)((cbase >> op.a) & 1ull);
            const C2 d = b ? d1 : d0;
#pragma unroll
            for (int j = 0; j < 16; j++) a[j] = cmul_r(a[j], d);
            break;
        }
        case SOP_DR: {
#pragma unroll
            for (int j = 0; j < 16; j++) a[j] = cmul_r(a[j], T.mats[op.idx + j]);
            break;
        }
        default:
            break;
        }
    }
    if (open) {
        if constexpr (sizeof(C2) == 16) {
            if (D != nullptr && D->okS) {
                const uint32_t x = s0s >> 4;
                const uint64_t base = cbase ^ D->sl[x & 63u] ^ D->sh[x >> 6];
#pragma unroll
                for (int j = 0; j < 16; j++) gst[base ^ D->sr[j]] = a[j];
                return;
            }
        }
        store_regs();
    }
}

}  // namespace
}  // namespace stage
}  // namespace kate
