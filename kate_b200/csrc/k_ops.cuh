// Shared-memory tile ops (any op kind, including dense blocks of up to 5
// qubits), used by the generic pass kernel and, between register stages, by
// the register-staged tile and batch kernels. The tile is stored
// XOR-swizzled: element i of a complex128 tile lives at swz(i), which
// spreads 16-byte accesses of lanes that differ in tile bits of distinct
// residue mod 3 over all banks. A complex64 tile uses swz2, which leaves bit
// 0 alone, so elements 2k and 2k + 1 stay side by side in one aligned
// 16-byte slot (one 16-byte copy moves both). Both maps are linear over
// GF(2) and are their own inverses.
// C2 is the tile's element type: double2 (FP64 arithmetic) or float2 (FP32);
// matrices always come from the FP64 pool.
#pragma once

#include "device_types.h"
#include "k_common.cuh"

namespace kate {
namespace ops {
namespace {

__host__ __device__ constexpr uint32_t swz(uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u); }
__host__ __device__ constexpr uint32_t swz2(uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 6u); }

// The swizzle of a tile of element type C2.
template <typename C2>
__host__ __device__ constexpr uint32_t tsw(uint32_t i) {
    return sizeof(C2) == 16 ? swz(i) : swz2(i);
}

template <int K, typename C2>
__device__ __forceinline__ void op_dense(C2* s, int m, const DevOp& op, const double2* __restrict__ mat, int tid, int nt) {
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
    for (uint32_t g = tid; g < groups; g += nt) {
        uint32_t base = g;
#pragma unroll
        for (int i = 0; i < K; i++) base = ins0(base, srt[i]);
        C2 x[D];
#pragma unroll
        for (int v = 0; v < D; v++) {
            uint32_t idx = base;
#pragma unroll
            for (int i = 0; i < K; i++)
                if ((v >> i) & 1) idx |= 1u << tb[i];
            x[v] = s[tsw<C2>(idx)];
        }
#pragma unroll
        for (int r = 0; r < D; r++) {
            C2 acc;
            acc.x = 0;
            acc.y = 0;
#pragma unroll
            for (int c = 0; c < D; c++) cfma(acc, from_pool<C2>(__ldg(mat + r * D + c)), x[c]);
            uint32_t idx = base;
#pragma unroll
            for (int i = 0; i < K; i++)
                if ((r >> i) & 1) idx |= 1u << tb[i];
            s[tsw<C2>(idx)] = acc;
        }
    }
}

// MAXK: widest dense op the caller can meet (wider ones are skipped; the
// host checks). Smaller values keep register use down.
template <typename C2, int MAXK = 5>
__device__ __noinline__ void apply_op(C2* s, int m, uint64_t base, const DevOp& op, const double2* __restrict__ pool,
                                      int tid, int nt) {
    using R = decltype(s->x);
    const uint32_t T = 1u << m;
    switch (op.kind) {
    case OPK_H: {
        const int t = op.tb[0];
        for (uint32_t p = tid; p < T / 2; p += nt) {
            uint32_t i0 = ins0(p, t), i1 = i0 | (1u << t);
            C2 a = s[tsw<C2>(i0)], b = s[tsw<C2>(i1)];
            C2 n0, n1;
            n0.x = (a.x + b.x) * (R)KATE_SQRT2INV;
            n0.y = (a.y + b.y) * (R)KATE_SQRT2INV;
            n1.x = n0.x - b.x * (R)KATE_SQRT2;
            n1.y = n0.y - b.y * (R)KATE_SQRT2;
            s[tsw<C2>(i0)] = n0;
            s[tsw<C2>(i1)] = n1;
        }
        break;
    }
    case OPK_X: {
        if ((base & op.pmask) != op.pmask) break;
        const int t = op.tb[0];
        for (uint32_t p = tid; p < T / 2; p += nt) {
            uint32_t i0 = ins0(p, t);
            if ((i0 & op.tmask) != op.tmask) continue;
            uint32_t i1 = i0 | (1u << t);
            C2 a = s[tsw<C2>(i0)];
            s[tsw<C2>(i0)] = s[tsw<C2>(i1)];
            s[tsw<C2>(i1)] = a;
        }
        break;
    }
    case OPK_PHASE: {
        if ((base & op.pmask) != op.pmask) break;
        C2 ph;
        ph.x = (R)op.ph_re;
        ph.y = (R)op.ph_im;
        for (uint32_t i = tid; i < T; i += nt)
            if ((i & op.tmask) == op.tmask) s[tsw<C2>(i)] = cmul(s[tsw<C2>(i)], ph);
        break;
    }
    case OPK_DIAG: {
        uint32_t cidx = 0;
        for (int i = 0; i < op.k; i++)
            if (op.ftb[i] < 0) cidx |= (uint32_t)((base >> op.fpos[i]) & 1ull) << i;
        const double2* tab = pool + op.mat;
        for (uint32_t x = tid; x < T; x += nt) {
            uint32_t d = cidx;
            for (int i = 0; i < op.k; i++)
                if (op.ftb[i] >= 0) d |= ((x >> op.ftb[i]) & 1u) << i;
            s[tsw<C2>(x)] = cmul(s[tsw<C2>(x)], from_pool<C2>(__ldg(tab + d)));
        }
        break;
    }
    case OPK_DENSE: {
        const double2* mat = pool + op.mat;
        switch (op.k) {
        case 1: op_dense<1>(s, m, op, mat, tid, nt); break;
        case 2: if (MAXK >= 2) op_dense<(MAXK >= 2 ? 2 : 1)>(s, m, op, mat, tid, nt); break;
        case 3: if (MAXK >= 3) op_dense<(MAXK >= 3 ? 3 : 1)>(s, m, op, mat, tid, nt); break;
        case 4: if (MAXK >= 4) op_dense<(MAXK >= 4 ? 4 : 1)>(s, m, op, mat, tid, nt); break;
        case 5: if (MAXK >= 5) op_dense<(MAXK >= 5 ? 5 : 1)>(s, m, op, mat, tid, nt); break;
        default: break;
        }
        break;
    }
    default:
        break;
    }
}

}  // namespace
}  // namespace ops
}  // namespace kate
