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

// Rank over GF(2) of four 4-bit columns.
int rank4(uint32_t c[4]) {
    int r = 0;
    for (int bit = 3; bit >= 0; bit--) {
        int piv = -1;
        for (int i = r; i < 4; i++)
            if ((c[i] >> bit) & 1u) piv = i;
        if (piv < 0) continue;
        std::swap(c[r], c[piv]);
        for (int i = 0; i < 4; i++)
            if (i != r && ((c[i] >> bit) & 1u)) c[i] ^= c[r];
        r++;
    }
    return r;
}

// Staging-tile swizzle of a pass (BlockProg::smask): v[b] is the 4-bit slot
// contribution of tile bit b >= 4 (bit k set: b is in smask[k]); tile bits
// 0..3 contribute their own unit vector. Each lane set (four tile bits whose
// values the 16 lanes of a half warp take) costs 2^(4 - rank) (the
// bank-pair conflict degree of its 8-byte accesses); coordinate descent from
// the fixed swizzle. smask[0] stays 0: amplitude pairs keep one 16-byte slot,
// so the tile is copied in 16-byte pieces (letting pairs split removed more
// conflicts but doubled the copy instructions and measured slower: 21.2
// against 22.5 layers/s on the 32-qubit brickwork).
void choose_swizzle(const std::vector<std::vector<int>>& sets, uint16_t smask[4]) {
    uint32_t v[KATE_TILE_BITS] = {0};
    for (int b = 4; b < KATE_TILE_BITS; b++) {
        // The fixed swizzle: bits 4..6 and 8..10 into slot bits 1..3.
        if (b >= 4 && b <= 6) v[b] = 2u << (b - 4);
        if (b >= 8 && b <= 10) v[b] = 2u << (b - 8);
    }
    auto col = [&](int b) { return b < 4 ? (1u << b) : v[b]; };
    auto cost = [&]() {
        int c = 0;
        for (const auto& st : sets) {
            uint32_t cc[4] = {col(st[0]), col(st[1]), col(st[2]), col(st[3])};
            c += 1 << (4 - rank4(cc));
        }
        return c;
    };
    int best = cost();
    for (int round = 0; round < 4; round++) {
        bool changed = false;
        for (int b = 4; b < KATE_TILE_BITS; b++) {
            uint32_t best_x = v[b];
            for (uint32_t x = 0; x < 16; x += 2) {  // slot bit 0 stays tile bit 0: pairs keep 16-byte copies
                v[b] = x;
                const int c = cost();
                if (c < best) {
                    best = c;
                    best_x = x;
                    changed = true;
                }
            }
            v[b] = best_x;
        }
        if (!changed) break;
    }
    for (int k = 0; k < 4; k++) {
        smask[k] = 0;
        for (int b = 4; b < KATE_TILE_BITS; b++)
            if ((v[b] >> k) & 1u) smask[k] |= (uint16_t)(1u << b);
    }
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
    // Lane sets: each block's rows (its 4 lowest non-block tile bits, the
    // lanes of a half warp in the A build and the read-back) and the
    // write-back's lanes (output tile bits 1..4 read the tile at input bits
    // outsrc[1..4]).
    std::vector<std::vector<int>> sets;
    for (int b = 0; b < nb; b++) {
        uint32_t bm = 0;
        for (int i = 0; i < 5; i++) bm |= 1u << out->btb[b][i];
        std::vector<int> st;
        for (int t = 0; t < m && st.size() < 4; t++)
            if (!((bm >> t) & 1u)) st.push_back(t);
        sets.push_back(st);
    }
    sets.push_back({out->outsrc[1], out->outsrc[2], out->outsrc[3], out->outsrc[4]});
    choose_swizzle(sets, out->smask);
    return "";
}

}  // namespace kate
