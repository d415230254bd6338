// Lowering of a complex64 pass into dense 5-qubit blocks for the tensor-core
// kernel (k_block_c64.cu). See BlockProg in device_types.h.
//
// The pass's gates, in program order, are merged greedily into blocks of at
// most five tile qubits (a block is the product of a contiguous run of the
// gate list, so no reordering is involved); each block's matrix is the FP64
// product from the gate merger (the reference's CPUmergeGate arithmetic),
// padded with identities to exactly five tile bits, then written as the
// real 64x64 operand in BF16 hi + lo parts (split-BF16 products: the kernel
// sums A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32).
#include <cmath>
#include <cstring>

#include "plan.hpp"

namespace kate {

namespace {

// BF16 bits of a float, rounded to nearest even (finite inputs).
uint16_t bf16_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
float bf16_value(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// Byte offset of element (row, k) in a K-major SWIZZLE_128B operand image of
// 64 BF16 columns: 128-byte rows, 16-byte chunks XORed with row & 7.
size_t sw128_offset_bf16(int row, int k) {
    const int chunk = k >> 3, w = k & 7;
    return (size_t)(row >> 3) * 1024 + (size_t)(row & 7) * 128 + (size_t)((chunk ^ (row & 7)) << 4) + (size_t)w * 2;
}

// The pass's gates as kate::Gate on tile-bit qubits.
bool tile_gate(const PGate& g, const std::vector<int>& tbit, Gate* out) {
    auto tb = [&](int q) { return tbit[q]; };
    Gate r;
    switch (g.kind) {
    case OPK_DENSE:
        r.id = G_DENSE;
        for (int q : g.tq) r.qbits.push_back(tb(q));
        r.dense = g.table;
        break;
    case OPK_H:
        r.id = G_H;
        r.qbits = {tb(g.tq[0])};
        break;
    case OPK_X:
        if (g.fq.size() == 1) {
            r.id = G_CNOT;
            r.qbits = {tb(g.tq[0]), tb(g.fq[0])};
        } else if (g.fq.size() == 2) {
            r.id = G_TOFFOLI;
            r.qbits = {tb(g.fq[0]), tb(g.fq[1]), tb(g.tq[0])};
        } else {
            return false;
        }
        break;
    case OPK_PHASE:
        r.id = G_DENSE;
        r.qbits = {tb(g.fq[0]), tb(g.fq[1])};
        r.dense.assign(16, Cx(0, 0));
        for (int i = 0; i < 3; i++) r.dense[i * 5] = Cx(1, 0);
        r.dense[15] = Cx(g.ph_re, g.ph_im);
        break;
    case OPK_DIAG: {
        r.id = G_DENSE;
        const int k = (int)g.fq.size(), dim = 1 << k;
        for (int q : g.fq) r.qbits.push_back(tb(q));
        r.dense.assign((size_t)dim * dim, Cx(0, 0));
        for (int i = 0; i < dim; i++) r.dense[(size_t)i * dim + i] = g.table[i];
        break;
    }
    default:
        return false;
    }
    for (int q : r.qbits)
        if (q < 0) return false;
    *out = std::move(r);
    return true;
}

}  // namespace

// Greedy block partition of `gates` (qubit sets): returns, for each gate,
// its block number.
std::vector<int> block_partition(const std::vector<PGate>& pg, const std::vector<int>& gates) {
    std::vector<int> which;
    uint64_t cur = 0;
    int blk = 0;
    for (size_t i = 0; i < gates.size(); i++) {
        const PGate& g = pg[gates[i]];
        uint64_t qs = 0;
        for (int q : g.tq) qs |= 1ull << q;
        for (int q : g.fq) qs |= 1ull << q;
        if (i > 0 && __builtin_popcountll(cur | qs) > 5) {
            blk++;
            cur = 0;
        }
        cur |= qs;
        which.push_back(blk);
    }
    return which;
}

std::string build_block_program(const Plan& plan, const PlannedPass& pass, int n, std::vector<uint8_t>& pool,
                                BlockProg* out) {
    const int m = (int)pass.phys_in.size();
    if (m != KATE_TILE_BITS) return "tensor-core blocks need 12-qubit tiles";
    std::memset(out, 0, sizeof(BlockProg));
    DevPass dp = to_devpass(n, pass, 0);
    out->m = m;
    out->ncb = dp.ncb;
    std::memcpy(out->tphys, dp.tphys, 16);
    std::memcpy(out->outsrc, dp.outsrc, 16);
    std::memcpy(out->cphys, dp.cphys, 48);
    std::vector<int> tbit(n, -1);
    for (int q = 0; q < n; q++)
        for (int t = 0; t < m; t++)
            if (pass.phys_in[t] == pass.phys_before[q]) tbit[q] = t;
    std::vector<int> which = block_partition(plan.pgates, pass.gates);
    const int nb = which.empty() ? 0 : which.back() + 1;
    if (nb < 1 || nb > KATE_C64_MAX_BLOCKS) return "pass has no block or too many blocks";
    out->nblocks = nb;
    for (int b = 0; b < nb; b++) {
        std::vector<Gate> gl;
        uint32_t used = 0;
        for (size_t i = 0; i < pass.gates.size(); i++) {
            if (which[i] != b) continue;
            Gate g;
            if (!tile_gate(plan.pgates[pass.gates[i]], tbit, &g)) return "gate outside the tile in a c64 pass";
            for (int q : g.qbits) used |= 1u << q;
            gl.push_back(std::move(g));
        }
        // Pad to exactly five tile bits with identities.
        for (int t = 0; t < m && __builtin_popcount(used) < 5; t++)
            if (!((used >> t) & 1u)) {
                Gate id;
                id.id = G_DENSE;
                id.qbits = {t};
                id.dense = {Cx(1, 0), Cx(0, 0), Cx(0, 0), Cx(1, 0)};
                gl.push_back(id);
                used |= 1u << t;
            }
        Gate U;
        std::string e = merge_gates(gl, &U);
        if (!e.empty()) return e;
        if (U.qbits.size() != 5) return "internal: block is not five qubits";
        for (int i = 0; i < 5; i++) out->btb[b][i] = (uint8_t)U.qbits[i];
        // Real form and its BF16 split, as K-major SWIZZLE_128B images.
        const size_t off = pool.size();
        pool.resize(off + KATE_BLOCK_IMG_BYTES, 0);
        uint8_t* hi_base = pool.data() + off;
        uint8_t* lo_base = pool.data() + off + KATE_BLOCK_IMG_BYTES / 2;
        for (int r = 0; r < 32; r++)
            for (int c = 0; c < 32; c++) {
                const Cx u = U.dense[(size_t)r * 32 + c];
                const double w[2][2] = {{u.re, -u.im}, {u.im, u.re}};
                for (int a = 0; a < 2; a++)
                    for (int bcol = 0; bcol < 2; bcol++) {
                        const int nrow = 2 * r + a, k = 2 * c + bcol;
                        const float f = (float)w[a][bcol];
                        const uint16_t h = bf16_bits(f);
                        const uint16_t l = bf16_bits(f - bf16_value(h));
                        const size_t o = sw128_offset_bf16(nrow, k);
                        std::memcpy(hi_base + o, &h, 2);
                        std::memcpy(lo_base + o, &l, 2);
                    }
            }
        out->bimg[b] = off;
    }
    return "";
}

}  // namespace kate
