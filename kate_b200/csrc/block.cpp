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
#include <algorithm>
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

// The FP64 product of a block's gates (at most five qubits) as a dense
// gate on the sorted union of their qubits. U starts as the identity and
// each gate multiplies it from the left, row group by row group, each step
// vectorised over U's 32 columns (the column-by-column gate merger costs
// several times more on the long blocks the light-cone selector forms).
// Not bit-identical to merge_gates (the operation order differs); the
// blocks are rounded to BF16 operands anyway.
std::string merge_block(const std::vector<Gate>& gl, Gate* out) {
    std::vector<int> cov;
    for (const Gate& g : gl) cov.insert(cov.end(), g.qbits.begin(), g.qbits.end());
    std::sort(cov.begin(), cov.end());
    cov.erase(std::unique(cov.begin(), cov.end()), cov.end());
    const int k = (int)cov.size();
    if (k > 5) return "internal: block wider than five qubits";
    const int dim = 1 << k;
    // Each gate as a local matrix; single-qubit gates are first multiplied
    // into a pending 2x2 per qubit, which the next wider gate on that qubit
    // absorbs (G' = G (x) pending, on G's column bit) or which is applied
    // alone at the end: on the light-cone blocks, which are mostly
    // rotations, U takes about a third of the row operations.
    struct LocalGate {
        int nq;
        int lb[5];
        size_t off;  // its matrix at mats[off], 2^nq x 2^nq
    };
    std::vector<LocalGate> ops;
    std::vector<Cx> mats;
    ops.reserve(gl.size());
    Cx Gbuf[32 * 32];
    Cx pend[5][4];
    bool has_pend[5] = {false, false, false, false, false};
    auto mul2 = [](const Cx* a, const Cx* b, Cx* r) {  // r = a b (2x2)
        Cx t[4];
        for (int x = 0; x < 2; x++)
            for (int y = 0; y < 2; y++) t[2 * x + y] = a[2 * x] * b[y] + a[2 * x + 1] * b[2 + y];
        for (int x = 0; x < 4; x++) r[x] = t[x];
    };
    for (const Gate& g : gl) {
        LocalGate L;
        L.nq = (int)g.qbits.size();
        const int gd = 1 << L.nq;
        for (int i = 0; i < L.nq; i++)
            L.lb[i] = (int)(std::lower_bound(cov.begin(), cov.end(), g.qbits[i]) - cov.begin());
        // The gate's own matrix, bit i of its index = qbits[i].
        Cx* G = Gbuf;
        for (int i = 0; i < gd * gd; i++) G[i] = Cx(0, 0);
        switch (g.id) {
        case G_DENSE:
            for (int i = 0; i < gd * gd; i++) G[i] = g.dense[i];
            break;
        case G_H: {
            const double h = 0.7071067811865475;
            G[0] = Cx(h, 0);
            G[1] = Cx(h, 0);
            G[2] = Cx(h, 0);
            G[3] = Cx(-h, 0);
            break;
        }
        case G_CNOT:  // qbits[0] flips when qbits[1] is 1
            G[0 * 4 + 0] = G[1 * 4 + 1] = Cx(1, 0);
            G[2 * 4 + 3] = G[3 * 4 + 2] = Cx(1, 0);
            break;
        case G_TOFFOLI:  // qbits[2] flips when qbits[0] and qbits[1] are 1
            for (int i = 0; i < 8; i++) G[i * 8 + i] = Cx(1, 0);
            G[3 * 8 + 3] = G[7 * 8 + 7] = Cx(0, 0);
            G[3 * 8 + 7] = G[7 * 8 + 3] = Cx(1, 0);
            break;
        case G_CRK: {
            const double t = ((double)2 * 3.1415926535897932384626433) / (double)(1ull << g.optarg);
            for (int i = 0; i < 3; i++) G[i * 4 + i] = Cx(1, 0);
            G[15] = Cx(std::cos(t), std::sin(t));
            break;
        }
        default:  // RX / RZ identifiers: no arithmetic, as in the reference
            for (int i = 0; i < gd; i++) G[i * gd + i] = Cx(1, 0);
            break;
        }
        if (L.nq == 1) {
            const int q = L.lb[0];
            if (has_pend[q]) mul2(G, pend[q], pend[q]);
            else for (int x = 0; x < 4; x++) pend[q][x] = G[x];
            has_pend[q] = true;
            continue;
        }
        // G' = G (I (x) P (x) I) for each pending P on the gate's bit i.
        for (int i = 0; i < L.nq; i++) {
            const int q = L.lb[i];
            if (!has_pend[q]) continue;
            const Cx* P = pend[q];
            for (int r = 0; r < gd; r++)
                for (int c0 = 0; c0 < gd; c0++) {
                    if ((c0 >> i) & 1) continue;
                    const int c1 = c0 | (1 << i);
                    const Cx g0 = G[r * gd + c0], g1 = G[r * gd + c1];
                    G[r * gd + c0] = g0 * P[0] + g1 * P[2];
                    G[r * gd + c1] = g0 * P[1] + g1 * P[3];
                }
            has_pend[q] = false;
        }
        L.off = mats.size();
        mats.insert(mats.end(), G, G + gd * gd);
        ops.push_back(L);
    }
    for (int q = 0; q < k; q++)
        if (has_pend[q]) {
            LocalGate L;
            L.nq = 1;
            L.lb[0] = q;
            L.off = mats.size();
            mats.insert(mats.end(), pend[q], pend[q] + 4);
            ops.push_back(L);
        }
    // U in separate real and imaginary planes (row-major), so the row
    // updates below vectorise.
    double ure[32 * 32], uim[32 * 32];
    for (int i = 0; i < dim * dim; i++) ure[i] = uim[i] = 0.0;
    for (int r = 0; r < dim; r++) ure[r * dim + r] = 1.0;
    double rre[32][32], rim[32][32];
    for (const LocalGate& L : ops) {
        const int nq = L.nq, gd = 1 << nq;
        const Cx* G = mats.data() + L.off;
        bool diag = true;
        for (int r = 0; r < gd && diag; r++)
            for (int c = 0; c < gd; c++)
                if (r != c && (G[r * gd + c].re != 0.0 || G[r * gd + c].im != 0.0)) {
                    diag = false;
                    break;
                }
        uint32_t tm = 0;
        for (int i = 0; i < nq; i++) tm |= 1u << L.lb[i];
        for (int base = 0; base < dim; base++) {
            if ((uint32_t)base & tm) continue;
            int idx[32];
            for (int s2 = 0; s2 < gd; s2++) {
                int x = base;
                for (int i = 0; i < nq; i++) x |= ((s2 >> i) & 1) << L.lb[i];
                idx[s2] = x;
            }
            if (diag) {  // scale each row
                for (int r = 0; r < gd; r++) {
                    const double ar = G[r * gd + r].re, ai = G[r * gd + r].im;
                    double* xr = ure + idx[r] * dim;
                    double* xi = uim + idx[r] * dim;
                    for (int c = 0; c < dim; c++) {
                        const double a = xr[c], b = xi[c];
                        xr[c] = ar * a - ai * b;
                        xi[c] = ar * b + ai * a;
                    }
                }
                continue;
            }
            for (int s2 = 0; s2 < gd; s2++)
                for (int c = 0; c < dim; c++) {
                    rre[s2][c] = ure[idx[s2] * dim + c];
                    rim[s2][c] = uim[idx[s2] * dim + c];
                }
            for (int r = 0; r < gd; r++) {
                double* xr = ure + idx[r] * dim;
                double* xi = uim + idx[r] * dim;
                for (int c = 0; c < dim; c++) xr[c] = xi[c] = 0.0;
                for (int s2 = 0; s2 < gd; s2++) {
                    const double ar = G[r * gd + s2].re, ai = G[r * gd + s2].im;
                    if (ar == 0.0 && ai == 0.0) continue;
                    const double* yr = rre[s2];
                    const double* yi = rim[s2];
                    for (int c = 0; c < dim; c++) {
                        xr[c] += ar * yr[c] - ai * yi[c];
                        xi[c] += ar * yi[c] + ai * yr[c];
                    }
                }
            }
        }
    }
    out->id = G_DENSE;
    out->qbits = cov;
    out->optarg = 0;
    out->dense.resize((size_t)dim * dim);
    for (int i = 0; i < dim * dim; i++) out->dense[i] = Cx(ure[i], uim[i]);
    return "";
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
        std::string e = merge_block(gl, &U);
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
