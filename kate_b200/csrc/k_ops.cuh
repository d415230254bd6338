// Shared-memory tile ops (any op kind, including dense blocks of up to 5
// qubits), used by the generic pass kernel and, between register stages, by
// the register-staged tile kernel. The tile is stored XOR-swizzled: element
// i lives at swz(i), which spreads 16-byte accesses of lanes that differ in
// tile bits of distinct residue mod 3 over all banks.
#pragma once

#include "device_types.h"
#include "k_common.cuh"

namespace kate {
namespace ops {
namespace {

__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u); }

template <int K>
__device__ __forceinline__ void op_dense(double2* s, int m, const DevOp& op, const double2* __restrict__ mat, int tid, int nt) {
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
        double2 x[D];
#pragma unroll
        for (int v = 0; v < D; v++) {
            uint32_t idx = base;
#pragma unroll
            for (int i = 0; i < K; i++)
                if ((v >> i) & 1) idx |= 1u << tb[i];
            x[v] = s[swz(idx)];
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
            s[swz(idx)] = acc;
        }
    }
}

__device__ __noinline__ void apply_op(double2* s, int m, uint64_t base, const DevOp& op, const double2* __restrict__ pool, int tid,
                         int nt) {
    const uint32_t T = 1u << m;
    switch (op.kind) {
    case OPK_H: {
        const int t = op.tb[0];
        for (uint32_t p = tid; p < T / 2; p += nt) {
            uint32_t i0 = ins0(p, t), i1 = i0 | (1u << t);
            double2 a = s[swz(i0)], b = s[swz(i1)];
            double2 n0 = make_double2((a.x + b.x) * KATE_SQRT2INV, (a.y + b.y) * KATE_SQRT2INV);
            s[swz(i0)] = n0;
            s[swz(i1)] = make_double2(n0.x - b.x * KATE_SQRT2, n0.y - b.y * KATE_SQRT2);
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
            double2 a = s[swz(i0)];
            s[swz(i0)] = s[swz(i1)];
            s[swz(i1)] = a;
        }
        break;
    }
    case OPK_PHASE: {
        if ((base & op.pmask) != op.pmask) break;
        const double2 ph = make_double2(op.ph_re, op.ph_im);
        for (uint32_t i = tid; i < T; i += nt)
            if ((i & op.tmask) == op.tmask) s[swz(i)] = cmul(s[swz(i)], ph);
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
            s[swz(x)] = cmul(s[swz(x)], __ldg(tab + d));
        }
        break;
    }
    case OPK_DENSE: {
        const double2* mat = pool + op.mat;
        switch (op.k) {
        case 1: op_dense<1>(s, m, op, mat, tid, nt); break;
        case 2: op_dense<2>(s, m, op, mat, tid, nt); break;
        case 3: op_dense<3>(s, m, op, mat, tid, nt); break;
        case 4: op_dense<4>(s, m, op, mat, tid, nt); break;
        case 5: op_dense<5>(s, m, op, mat, tid, nt); break;
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
