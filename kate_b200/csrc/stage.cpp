// Lowering of a planned pass into the register-staged program run by the
// tile kernel (k_tile.cu). See device_types.h for the program format.
//
// The pass's ops are list-scheduled into stages. A stage fixes four tile
// bits as register bits; ops whose target is one of them (2x2, H, X) or
// that have no target (controlled phase, one-qubit diagonal) are applied to
// registers. Ops are reordered only across ops that share no qubit, so the
// result is unchanged. Each stage boundary costs one round trip of the tile
// through shared memory, so the scheduler first takes ready ops whose target
// is already a register bit, then grows the register set (up to four bits),
// and closes the stage only when neither is possible.
#include <cmath>
#include <algorithm>
#include <cstring>

#include "plan.hpp"

namespace kate {

namespace {

struct LOp {
    int kind = 0;        // SOP_*
    int tgt = -1;        // target tile bit
    int tgt2 = -1;       // U2: second target tile bit (matrix index bit 1)
    Cx m2[16];           // U2: 4x4 matrix, row-major
    uint32_t tctl = 0;   // control tile bits
    uint64_t pctl = 0;   // control coset (physical) bits
    int dtile = -1;      // D1: tile bit, or -1
    int dphys = -1;      // D1: physical bit when outside the tile
    Cx m[4];
    int smem = -1;       // SMEM: index into smem_ops
    std::vector<int> qs; // logical qubits (dependencies)
};

bool is_one(Cx v) { return v.re == 1.0 && v.im == 0.0; }

Cx cdiv(Cx a, Cx b) {
    const double d = b.re * b.re + b.im * b.im;
    return Cx((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

// Multiplicative Moebius transform of a 2^k diagonal table: h[S] with
// table[b] = prod over S subset of b of h[S]. False (h untouched) when an
// entry is zero or k is outside 2..5.
bool diag_factors(const std::vector<Cx>& table, int k, std::vector<Cx>* h) {
    if (k < 2 || k > 5 || table.size() != (1u << k)) return false;
    for (const Cx& v : table)
        if (v.re == 0.0 && v.im == 0.0) return false;
    if (!h) return true;
    *h = table;
    for (int i = 0; i < k; i++)
        for (uint32_t S = 0; S < (1u << k); S++)
            if ((S >> i) & 1u) (*h)[S] = cdiv((*h)[S], (*h)[S & ~(1u << i)]);
    return true;
}

}  // namespace

// Rewrites real and RX-form 2x2 ops whose matrix is a common factor f times
// a matrix with a unit entry in each row (SOP_URA/URB/UXA/UXB), picking the
// factor of larger magnitude so that |t0|, |t1| <= 1, and applies the
// product F of the factors once: F multiplies the entries of the pass's
// first diagonal (DR, D1) or general 2x2 (U) op, or, when the pass has none,
// the first rewritten op goes back to a general 2x2 carrying F.
void scale_rotations(std::vector<SOp>& ops, std::vector<Cx>& mats) {
    Cx F(1.0, 0.0);
    int first = -1;
    std::vector<Cx> orig;  // matrix of the first rewritten op
    for (size_t k = 0; k < ops.size(); k++) {
        SOp& o = ops[k];
        if (o.kind != SOP_UR && o.kind != SOP_UX) continue;
        const Cx* m = &mats[o.idx];
        double a, b, c, d;
        const bool ux = o.kind == SOP_UX;
        if (ux) {
            a = m[0].re, b = m[1].im, c = m[2].im, d = m[3].re;
        } else {
            a = m[0].re, b = m[1].re, c = m[2].re, d = m[3].re;
        }
        const bool formA = a == d && a != 0.0;
        const bool formB = b != 0.0 && (ux ? c == b : c == -b);
        if (!formA && !formB) continue;
        const bool useA = formA && (!formB || std::fabs(a) >= std::fabs(b));
        if (first < 0) {
            first = (int)k;
            orig.assign(m, m + 4);
        }
        Cx f, t;
        if (useA) {
            f = Cx(a, 0.0);
            t = Cx(b / a, c / a);
            o.kind = ux ? SOP_UXA : SOP_URA;
        } else {
            f = ux ? Cx(0.0, b) : Cx(b, 0.0);
            t = Cx(a / b, d / b);
            o.kind = ux ? SOP_UXB : SOP_URB;
        }
        F = F * f;
        // The op keeps its 4-entry slot; entry 0 holds (t0, t1), entry 1 the factor.
        mats[o.idx] = t;
        mats[o.idx + 1] = f;
    }
    if (first < 0) return;
    for (SOp& o : ops) {
        int cnt = o.kind == SOP_DR ? 16 : o.kind == SOP_D1 ? 2 : o.kind == SOP_U ? 4 : 0;
        if (!cnt) continue;
        for (int i = 0; i < cnt; i++) mats[o.idx + i] = mats[o.idx + i] * F;
        return;
    }
    // No op to absorb F: the first rewritten op becomes a general 2x2 with
    // its own factor replaced by F.
    SOp& o = ops[first];
    const Cx f = mats[o.idx + 1];
    // G = F / f (f is real or purely imaginary and nonzero).
    const double n2 = f.re * f.re + f.im * f.im;
    const Cx G = F * Cx(f.re / n2, -f.im / n2);
    for (int i = 0; i < 4; i++) mats[o.idx + i] = orig[i] * G;
    o.kind = SOP_U;
}

int classify_2x2(const Cx* m) {
    bool real = true, rx = true;
    for (int i = 0; i < 4; i++) real &= m[i].im == 0.0;
    rx = m[0].im == 0.0 && m[3].im == 0.0 && m[1].re == 0.0 && m[2].re == 0.0;
    return real ? SOP_UR : rx ? SOP_UX : SOP_U;
}

int prog_round_trips(const PassProg& p) {
    if (p.nstages <= 0) return 0;
    int r = p.nstages - 1;
    for (int i = 0; i < 4; i++)
        if (p.srb[0][i] < 4) {
            r++;
            break;
        }
    const int l = p.nstages - 1;
    uint32_t want = 0, have = 0;
    for (int i = 0; i < 4; i++) want |= 1u << p.outsrc[i], have |= 1u << p.stb[l][i];
    return r + (want != have ? 1 : 0);
}

std::string build_pass_program(const Plan& plan, const PlannedPass& pass, int n, std::vector<DevOp>& smem_ops,
                               std::vector<Cx>& pool, PassProg* out, bool dense2, bool low_first) {
    const int m = (int)pass.phys_in.size();
    if (m != KATE_TILE_BITS) return "register-staged kernel needs 12-qubit tiles";
    const std::vector<int>& phys = pass.phys_before;
    const int sop_begin = (int)smem_ops.size();
    auto tile_bit = [&](int q) -> int {
        int p = phys[q];
        for (int t = 0; t < m; t++)
            if (pass.phys_in[t] == p) return t;
        return -1;
    };
    std::vector<LOp> L;
    for (int gi : pass.gates) {
        const PGate& g = plan.pgates[gi];
        LOp o;
        o.qs = g.tq;
        o.qs.insert(o.qs.end(), g.fq.begin(), g.fq.end());
        auto controls = [&]() {
            for (int q : g.fq) {
                int t = tile_bit(q);
                if (t >= 0) o.tctl |= 1u << t;
                else o.pctl |= 1ull << phys[q];
            }
        };
        if (g.kind == OPK_DENSE && g.tq.size() == 1) {
            o.kind = classify_2x2(g.table.data());
            o.tgt = tile_bit(g.tq[0]);
            for (int i = 0; i < 4; i++) o.m[i] = g.table[i];
        } else if (g.kind == OPK_DENSE && g.tq.size() == 2 && dense2) {
            o.kind = SOP_U2;
            o.tgt = tile_bit(g.tq[0]);
            o.tgt2 = tile_bit(g.tq[1]);
            for (int i = 0; i < 16; i++) o.m2[i] = g.table[i];
            if (o.tgt2 < 0) return "internal: target outside the tile";
        } else if (g.kind == OPK_H) {
            o.kind = SOP_H;
            o.tgt = tile_bit(g.tq[0]);
        } else if (g.kind == OPK_X) {
            o.kind = SOP_X;
            o.tgt = tile_bit(g.tq[0]);
            controls();
        } else if (g.kind == OPK_PHASE) {
            o.kind = SOP_PH;
            controls();
            o.m[0] = Cx(g.ph_re, g.ph_im);
        } else if (g.kind == OPK_DIAG && g.fq.size() == 1) {
            o.kind = SOP_D1;
            o.dtile = tile_bit(g.fq[0]);
            if (o.dtile < 0) o.dphys = phys[g.fq[0]];
            o.m[0] = g.table[0];
            o.m[1] = g.table[1];
        } else if (g.kind == OPK_DIAG && diag_factors(g.table, (int)g.fq.size(), nullptr)) {
            // A k-qubit diagonal as register ops: its multiplicative Moebius
            // factors h[S] (table[b] = product of h[S] over the bit sets S
            // contained in b) become one-qubit diagonals (|S| = 1, with h[{}]
            // folded into the first) and controlled phases on the qubits of S.
            const int k = (int)g.fq.size();
            std::vector<Cx> h;
            diag_factors(g.table, k, &h);
            bool first = true;
            for (uint32_t S = 1; S < (1u << k); S++) {
                const int pc = __builtin_popcount(S);
                Cx v = h[S];
                if (pc == 1) {
                    const int i = __builtin_ctz(S);
                    const Cx d0 = first ? h[0] : Cx(1.0, 0.0);
                    const Cx d1 = first ? h[0] * v : v;
                    first = false;
                    if (is_one(d0) && is_one(d1)) continue;
                    LOp d;
                    d.kind = SOP_D1;
                    d.dtile = tile_bit(g.fq[i]);
                    if (d.dtile < 0) d.dphys = phys[g.fq[i]];
                    d.m[0] = d0;
                    d.m[1] = d1;
                    d.qs = {g.fq[i]};
                    L.push_back(std::move(d));
                } else {
                    if (is_one(v)) continue;
                    LOp c;
                    c.kind = SOP_PH;
                    c.m[0] = v;
                    for (int i = 0; i < k; i++)
                        if ((S >> i) & 1u) {
                            const int q = g.fq[i];
                            const int t = tile_bit(q);
                            if (t >= 0) c.tctl |= 1u << t;
                            else c.pctl |= 1ull << phys[q];
                            c.qs.push_back(q);
                        }
                    L.push_back(std::move(c));
                }
            }
            continue;
        } else {
            o.kind = SOP_SMEM;
            PlannedPass one;
            one.phys_in = pass.phys_in;
            one.gates = {gi};
            lower_pass(plan, one, phys, pool);
            o.smem = (int)smem_ops.size();
            smem_ops.push_back(one.ops[0]);
        }
        if ((o.kind == SOP_U || o.kind == SOP_UR || o.kind == SOP_UX || o.kind == SOP_H || o.kind == SOP_X ||
             o.kind == SOP_U2) &&
            o.tgt < 0)
            return "internal: target outside the tile";
        L.push_back(std::move(o));
    }
    const int N = (int)L.size();
    // Dependencies: the previous op touching any of the same qubits.
    std::vector<std::vector<int>> preds(N);
    {
        std::vector<int> last(n, -1);
        for (int i = 0; i < N; i++) {
            for (int q : L[i].qs)
                if (last[q] >= 0) preds[i].push_back(last[q]);
            for (int q : L[i].qs) last[q] = i;
        }
    }
    std::vector<char> done(N, 0);
    auto ready = [&](int i, const std::vector<char>& d) {
        if (d[i]) return false;
        for (int p : preds[i])
            if (!d[p]) return false;
        return true;
    };
    auto regable = [&](int i) { return L[i].kind != SOP_SMEM; };

    std::memset(out, 0, sizeof(PassProg));
    DevPass dp = to_devpass(n, pass, 0);
    out->m = m;
    out->ncb = dp.ncb;
    std::memcpy(out->tphys, dp.tphys, 16);
    std::memcpy(out->outsrc, dp.outsrc, 16);
    std::memcpy(out->cphys, dp.cphys, 48);
    out->sop0 = sop_begin;
    std::vector<SOp> ops;
    std::vector<Cx> mats;

    // Greedy register stage from the ops not yet done: its register bits R
    // (at most 4 targets) and its op list in order.
    // Each pick is the lowest-index ready op whose target is a register bit
    // (or that has none), else the lowest-index ready op with a target while
    // R has room. The ready ops are kept as an ascending list, updated from
    // the pending-predecessor counts as ops are picked.
    std::vector<std::vector<int>> succs(N);
    for (int i = 0; i < N; i++)
        for (int p : preds[i]) succs[p].push_back(i);
    std::vector<int> npend(N);
    auto select = [&](const std::vector<char>& base, std::vector<int>& R, std::vector<int>& list, uint32_t avoid) {
        std::vector<int> rdy;
        for (int i = 0; i < N; i++) {
            int c = 0;
            for (int p : preds[i]) c += !base[p];
            npend[i] = c;
            if (!base[i] && c == 0) rdy.push_back(i);
        }
        auto in_R = [&](int t) { return std::find(R.begin(), R.end(), t) != R.end(); };
        // Targets of op i not yet register bits (-1 entries ignored).
        auto missing = [&](int i) {
            int c = 0;
            if (L[i].tgt >= 0 && !in_R(L[i].tgt)) c++;
            if (L[i].tgt2 >= 0 && !in_R(L[i].tgt2)) c++;
            return c;
        };
        for (;;) {
            size_t at = rdy.size();
            for (size_t k = 0; k < rdy.size() && at == rdy.size(); k++) {
                const int i = rdy[k];
                if (regable(i) && missing(i) == 0) at = k;
            }
            if (at == rdy.size() && R.size() < 4)
                for (size_t k = 0; k < rdy.size() && at == rdy.size(); k++) {
                    const int i = rdy[k];
                    const bool avoided = (L[i].tgt >= 0 && !in_R(L[i].tgt) && ((avoid >> L[i].tgt) & 1u)) ||
                                         (L[i].tgt2 >= 0 && !in_R(L[i].tgt2) && ((avoid >> L[i].tgt2) & 1u));
                    if (regable(i) && L[i].tgt >= 0 && R.size() + missing(i) <= 4 && !avoided) {
                        at = k;
                        if (!in_R(L[i].tgt)) R.push_back(L[i].tgt);
                        if (L[i].tgt2 >= 0 && !in_R(L[i].tgt2)) R.push_back(L[i].tgt2);
                    }
                }
            if (at == rdy.size()) break;
            const int pick = rdy[at];
            rdy.erase(rdy.begin() + (long)at);
            list.push_back(pick);
            for (int s : succs[pick])
                if (--npend[s] == 0 && !base[s]) rdy.insert(std::lower_bound(rdy.begin(), rdy.end(), s), s);
        }
    };
    auto pad = [&](std::vector<int>& R, uint32_t avoid) {
        for (int pass2 = 0; pass2 < 2; pass2++)
            for (int t = 0; t < m && R.size() < 4; t++)
                if ((pass2 == 1 || !((avoid >> t) & 1u)) && std::find(R.begin(), R.end(), t) == R.end())
                    R.push_back(t);
    };
    // Warp bits (thread bits 5..7) of the previous stage, when its registers
    // are still open (no shared-memory op since): a stage that keeps them,
    // on tile bits outside both stages' registers, exchanges the tile only
    // within each warp (every warp stores and reloads the slots whose warp
    // bits are its index), so its boundary needs a warp barrier only.
    std::vector<int> prevW;
    bool prev_open = false;

    int scheduled = 0;
    while (scheduled < N) {
        // Tentative register stage.
        std::vector<int> R, list;
        uint32_t avoid = low_first && out->nstages == 0 ? 0xFu : 0u;
        select(done, R, list, avoid);
        if (list.empty() && avoid) {
            avoid = 0;
            R.clear();
            select(done, R, list, avoid);
        }
        if (list.empty()) {
            int first = -1;
            for (int i = 0; i < N && first < 0; i++)
                if (ready(i, done)) first = i;
            if (first < 0 || regable(first)) return "internal: stage scheduler stalled";
            SOp s{};
            s.kind = SOP_SMEM;
            s.idx = (uint16_t)(L[first].smem - out->sop0);
            ops.push_back(s);
            done[first] = 1;
            scheduled++;
            prev_open = false;
            continue;
        }
        pad(R, avoid);
        std::vector<int> nonR;
        for (int t = 0; t < m; t++)
            if (std::find(R.begin(), R.end(), t) == R.end()) nonR.push_back(t);
        auto is_nonR = [&](int t) { return std::find(nonR.begin(), nonR.end(), t) != nonR.end(); };
        // Warp bits: the previous stage's when they are not register bits
        // here (warp-local boundary), else three non-register bits that the
        // next stage (looked ahead) does not take as registers either. Only
        // bits above 3 qualify while there are enough: tile bits 0..3 are
        // physical bits 0..3 and stay lanes, which keeps the first and last
        // stages' HBM accesses in 256-byte runs (worth more than a warp-local
        // boundary).
        // The bits that must stay lanes 0..3: the first stage's loads read
        // HBM in 256-byte runs when tile bits 0..3 (physical bits 0..3) are
        // its lanes 0..3, and the last stage's stores write them when the
        // tile bits that the write-back moves to physical bits 0..3
        // (outsrc[0..3]) are. Other stages keep tile bits 0..3 off the warps.
        const bool first_stage = out->nstages == 0;
        const bool last_stage = scheduled + (int)list.size() == N;
        uint32_t lowset = 0xFu;
        if (last_stage && !first_stage) {
            lowset = 0;
            for (int i = 0; i < 4; i++) lowset |= 1u << out->outsrc[i];
        }
        auto is_low = [&](int t) { return ((lowset >> t) & 1u) != 0; };
        bool local_in = prev_open && prevW.size() == 3;
        for (int t : prevW)
            if (!is_nonR(t) || is_low(t)) local_in = false;
        std::vector<int> Wb;
        if (local_in) {
            Wb = prevW;
        } else {
            std::vector<char> dn(done);
            for (int i : list) dn[i] = 1;
            std::vector<int> Rn, ln;
            select(dn, Rn, ln, 0);
            if (!ln.empty()) pad(Rn, 0);
            auto in_Rn = [&](int t) { return std::find(Rn.begin(), Rn.end(), t) != Rn.end(); };
            for (int pass2 = 0; pass2 < 3 && Wb.size() < 3; pass2++)
                for (int k = (int)nonR.size() - 1; k >= 0 && Wb.size() < 3; k--) {
                    const int t = nonR[k];
                    if (std::find(Wb.begin(), Wb.end(), t) != Wb.end()) continue;
                    const bool ok = pass2 == 0 ? (!is_low(t) && !in_Rn(t)) : pass2 == 1 ? !is_low(t) : true;
                    if (ok) Wb.push_back(t);
                }
        }
        auto in_R = [&](int t) { return std::find(R.begin(), R.end(), t) != R.end(); };
        // NOTs/CNOTs folded into addressing. An X is foldable when its
        // controls are either one register bit or only thread/coset bits.
        // It joins the load prefix when it commutes with every op kept in the
        // stage before it, and the store suffix when it commutes with every
        // kept op after it. Ops commute when neither's target is a qubit the
        // other touches (controls and diagonals only read the Z basis).
        auto targets = [&](const LOp& o) {
            uint32_t m2 = 0;
            if (o.tgt >= 0) m2 |= 1u << o.tgt;
            if (o.tgt2 >= 0) m2 |= 1u << o.tgt2;
            return m2;
        };
        auto touched = [&](const LOp& o) {
            uint32_t m2 = o.tctl | targets(o);
            if (o.dtile >= 0) m2 |= 1u << o.dtile;
            return m2;
        };
        auto commute = [&](const LOp& a, const LOp& b) {
            return !(targets(a) & touched(b)) && !(targets(b) & touched(a));
        };
        auto reg_ctl = [&](const LOp& o) {
            return o.pctl == 0 && __builtin_popcount(o.tctl) == 1 && in_R(__builtin_ctz(o.tctl));
        };
        auto lane_ctl = [&](const LOp& o) {
            for (int t = 0; t < m; t++)
                if (((o.tctl >> t) & 1u) && in_R(t)) return false;
            return true;  // includes the uncontrolled NOT
        };
        auto foldable = [&](const LOp& o) { return o.kind == SOP_X && (reg_ctl(o) || lane_ctl(o)); };
        std::vector<int> prefix, kept;
        for (int i : list) {
            bool ok = foldable(L[i]);
            for (int k : kept)
                if (ok && !commute(L[k], L[i])) ok = false;
            (ok ? prefix : kept).push_back(i);
        }
        std::vector<int> suffix;
        for (int ki = (int)kept.size() - 1; ki >= 0; ki--) {
            const int i = kept[ki];
            bool ok = foldable(L[i]);
            for (size_t k2 = ki + 1; k2 < kept.size() && ok; k2++)
                if (std::find(suffix.begin(), suffix.end(), kept[k2]) == suffix.end() &&
                    !commute(L[i], L[kept[k2]]))
                    ok = false;
            if (ok) suffix.insert(suffix.begin(), i);
        }
        std::vector<int> body;
        for (int i : kept)
            if (std::find(suffix.begin(), suffix.end(), i) == suffix.end()) body.push_back(i);
        // Thread map: lanes first — three low thread bits (the lanes of one
        // quarter-warp phase of a 16-byte shared-memory access) on tile bits
        // of distinct residue mod 3 (distinct bank groups under the XOR
        // swizzle of the tile), then the other lane bits ascending — then
        // the warp bits. Among such triples the one with the fewest control
        // bits of NOTs folded into this stage's loads or stores is taken: a
        // flip conditioned on a phase lane moves only some of the phase's
        // addresses and can put two of them in one bank group. The first
        // and the last stage keep their low bits (above) on lanes 0..3 for
        // their 256-byte HBM runs.
        uint32_t flipctl = 0;
        for (int i : prefix)
            if (!reg_ctl(L[i])) flipctl |= L[i].tctl;
        for (int i : suffix)
            if (!reg_ctl(L[i])) flipctl |= L[i].tctl;
        std::vector<int> lanes, tb;
        for (int t : nonR)
            if (std::find(Wb.begin(), Wb.end(), t) == Wb.end()) lanes.push_back(t);
        const bool edge = first_stage || last_stage;
        bool low4 = edge;
        for (int t = 0; t < m && low4; t++)
            if (is_low(t) && std::find(lanes.begin(), lanes.end(), t) == lanes.end()) low4 = false;
        int best = -1, bt[3] = {-1, -1, -1};
        const int nl = (int)lanes.size();
        for (int x = 0; x < nl; x++)
            for (int y = x + 1; y < nl; y++)
                for (int z = y + 1; z < nl; z++) {
                    const int a = lanes[x], b2 = lanes[y], c2 = lanes[z];
                    if (a % 3 == b2 % 3 || a % 3 == c2 % 3 || b2 % 3 == c2 % 3) continue;
                    if (low4 && !(is_low(a) && is_low(b2) && is_low(c2))) continue;
                    const int cost = (int)((flipctl >> a) & 1u) + (int)((flipctl >> b2) & 1u) + (int)((flipctl >> c2) & 1u);
                    if (best < 0 || cost < best) best = cost, bt[0] = a, bt[1] = b2, bt[2] = c2;
                }
        if (best >= 0) {
            for (int i = 0; i < 3; i++) tb.push_back(bt[i]);
        } else if (low4) {
            // No triple of distinct bank groups among the low bits: the
            // 256-byte runs come first.
            for (int t : lanes)
                if (is_low(t)) tb.push_back(t);
        } else {
            bool res_used[3] = {false, false, false};
            for (int t : lanes)
                if (tb.size() < 3 && !res_used[t % 3]) {
                    res_used[t % 3] = true;
                    tb.push_back(t);
                }
        }
        if (low4)
            for (int t : lanes)
                if (is_low(t) && std::find(tb.begin(), tb.end(), t) == tb.end()) tb.push_back(t);
        for (int t : lanes)
            if (std::find(tb.begin(), tb.end(), t) == tb.end()) tb.push_back(t);
        for (int t : Wb) tb.push_back(t);
        prevW = Wb;
        prev_open = true;
        auto regpos = [&](int t) { return (int)(std::find(R.begin(), R.end(), t) - R.begin()); };
        auto thrpos = [&](int t) { return (int)(std::find(tb.begin(), tb.end(), t) - tb.begin()); };
        if (out->nstages >= KATE_MAX_STAGES) return "pass program has too many stages";
        const int si = out->nstages++;
        for (int i = 0; i < 4; i++) out->srb[si][i] = (uint8_t)R[i];
        for (int i = 0; i < 8; i++) out->stb[si][i] = (uint8_t)tb[i];
        uint16_t* stab = out->stab[si];
        auto swz = [](uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u); };
        for (int v = 0; v < 16; v++) {
            uint32_t lo = 0, hi = 0;
            for (int i = 0; i < 4; i++) {
                if ((v >> i) & 1) lo |= 1u << tb[i];
                if ((v >> i) & 1) hi |= 1u << tb[4 + i];
            }
            stab[v] = (uint16_t)(swz(lo) << 4);
            stab[16 + v] = (uint16_t)(swz(hi) << 4);
        }
        uint32_t wnat[4];
        for (int i = 0; i < 4; i++) wnat[i] = swz(1u << R[i]) << 4;
        auto W = [&](uint32_t x) {
            uint32_t r = 0;
            for (int k = 0; k < 4; k++)
                if ((x >> k) & 1u) r ^= wnat[k];
            return r;
        };


        // Affine map x -> M x ^ sum_k g_k u_k of a folded X sequence on the
        // 4-bit register index: register CNOTs update M (and the lane vectors
        // already accumulated), lane NOTs add u = e_B with their condition g.
        struct Lane {
            uint32_t u;
            uint8_t cthr;
            uint64_t ccos;
        };
        auto compose = [&](const std::vector<int>& seq, uint32_t col[4], std::vector<Lane>& lanes) {
            for (int i = 0; i < 4; i++) col[i] = 1u << i;
            for (int i : seq) {
                const LOp& o = L[i];
                const int B = regpos(o.tgt);
                if (reg_ctl(o)) {
                    const int C = regpos(__builtin_ctz(o.tctl));
                    for (int k = 0; k < 4; k++) col[k] ^= ((col[k] >> C) & 1u) << B;
                    for (auto& ln : lanes) ln.u ^= ((ln.u >> C) & 1u) << B;
                } else {
                    Lane ln{1u << B, 0, o.pctl};
                    for (int t = 0; t < m; t++)
                        if ((o.tctl >> t) & 1u) ln.cthr |= (uint8_t)(1u << thrpos(t));
                    lanes.push_back(ln);
                }
            }
        };
        auto apply = [](const uint32_t col[4], uint32_t x) {
            uint32_t r = 0;
            for (int k = 0; k < 4; k++)
                if ((x >> k) & 1u) r ^= col[k];
            return r;
        };
        // Load fold: register j must receive the amplitude at pi^-1(j).
        uint32_t pcol[4];
        std::vector<Lane> plane;
        compose(prefix, pcol, plane);
        uint32_t inv[16];
        for (uint32_t x = 0; x < 16; x++) inv[apply(pcol, x)] = x;
        std::vector<SOp> xl;
        for (auto& ln : plane) {
            SOp f{};
            f.kind = SOP_XL;
            f.cthr = ln.cthr;
            f.ccos = ln.ccos;
            f.idx = (uint16_t)W(inv[ln.u]);
            xl.push_back(f);
        }
        for (int i = 0; i < 4; i++) stab[32 + i] = (uint16_t)W(inv[1u << i]);
        // Store fold: register j (natural index j) goes to pi(j).
        uint32_t scol[4];
        std::vector<Lane> slane;
        compose(suffix, scol, slane);
        std::vector<SOp> folds;
        for (auto& ln : slane) {
            SOp f{};
            f.kind = SOP_XF;
            f.cthr = ln.cthr;
            f.ccos = ln.ccos;
            f.idx = (uint16_t)W(ln.u);
            folds.push_back(f);
        }
        for (int i = 0; i < 4; i++) stab[36 + i] = (uint16_t)W(scol[i]);
        for (int i = 0; i < 4; i++) stab[40 + i] = (uint16_t)wnat[i];

        ops.insert(ops.end(), xl.begin(), xl.end());
        SOp st{};
        st.kind = SOP_STAGE;
        st.idx = (uint16_t)si;
        st.src = local_in ? 1 : 0;  // boundary needs a warp barrier only
        ops.push_back(st);
        for (int i : prefix) done[i] = 1;
        for (int i : suffix) done[i] = 1;
        scheduled += (int)(prefix.size() + suffix.size());
        list = body;
        auto ctl = [&](const LOp& o, SOp& s) {
            for (int t = 0; t < m; t++)
                if ((o.tctl >> t) & 1u) {
                    int r = regpos(t);
                    if (r < 4) s.creg |= (uint8_t)(1u << r);
                    else s.cthr |= (uint8_t)(1u << thrpos(t));
                }
            s.ccos = o.pctl;
        };
        // Diagonals over register bits (one-qubit diagonals, phases whose
        // controls are all register bits) are multiplied into one pending
        // 16-entry table and emitted as a single op just before the first op
        // that targets one of the bits it depends on (they commute with
        // everything else), or at the end of the stage.
        Cx dr[16];
        uint32_t dr_support = 0;
        auto dr_reset = [&]() {
            for (auto& v : dr) v = Cx(1.0, 0.0);
            dr_support = 0;
        };
        auto dr_flush = [&]() {
            if (!dr_support) return;
            SOp f{};
            f.kind = SOP_DR;
            f.idx = (uint16_t)mats.size();
            mats.insert(mats.end(), dr, dr + 16);
            ops.push_back(f);
            dr_reset();
        };
        dr_reset();
        for (int i : list) {
            const LOp& o = L[i];
            SOp s{};
            s.kind = (uint8_t)o.kind;
            if (o.tgt >= 0 && dr_support && ((dr_support >> regpos(o.tgt)) & 1u)) dr_flush();
            if (o.tgt2 >= 0 && dr_support && ((dr_support >> regpos(o.tgt2)) & 1u)) dr_flush();
            switch (o.kind) {
            case SOP_U2: {
                // Register bits a < src; with the targets the other way round
                // the matrix's index bits 0 and 1 trade places.
                int r0 = regpos(o.tgt), r1 = regpos(o.tgt2);
                const bool swap = r0 > r1;
                s.a = (uint8_t)(swap ? r1 : r0);
                s.src = (uint8_t)(swap ? r0 : r1);
                s.idx = (uint16_t)mats.size();
                auto sw = [&](int v) { return swap ? (((v & 1) << 1) | ((v >> 1) & 1)) : v; };
                for (int r = 0; r < 4; r++)
                    for (int c = 0; c < 4; c++) mats.push_back(o.m2[4 * sw(r) + sw(c)]);
                break;
            }
            case SOP_U:
            case SOP_UR:
            case SOP_UX:
                s.a = (uint8_t)regpos(o.tgt);
                s.idx = (uint16_t)mats.size();
                mats.insert(mats.end(), o.m, o.m + 4);
                break;
            case SOP_H:
                s.a = (uint8_t)regpos(o.tgt);
                break;
            case SOP_X:
                s.a = (uint8_t)regpos(o.tgt);
                ctl(o, s);
                break;
            case SOP_PH:
                ctl(o, s);
                if (s.cthr == 0 && s.ccos == 0) {
                    for (int j = 0; j < 16; j++)
                        if (((uint32_t)j & s.creg) == s.creg) dr[j] = dr[j] * o.m[0];
                    dr_support |= s.creg ? s.creg : 1u;
                    s.kind = 0;
                    break;
                }
                s.idx = (uint16_t)mats.size();
                mats.push_back(o.m[0]);
                break;
            case SOP_D1:
                if (o.dtile >= 0) {
                    int r = regpos(o.dtile);
                    if (r < 4) {
                        for (int j = 0; j < 16; j++) dr[j] = dr[j] * o.m[(j >> r) & 1];
                        dr_support |= 1u << r;
                        s.kind = 0;
                        break;
                    }
                    s.src = SRC_THR;
                    s.a = (uint8_t)thrpos(o.dtile);
                } else {
                    s.src = SRC_COS;
                    s.a = (uint8_t)o.dphys;
                }
                s.idx = (uint16_t)mats.size();
                mats.push_back(o.m[0]);
                mats.push_back(o.m[1]);
                break;
            default:
                return "internal: unexpected op in a register stage";
            }
            if (s.kind) ops.push_back(s);
            done[i] = 1;
            scheduled++;
        }
        dr_flush();
        ops.insert(ops.end(), folds.begin(), folds.end());
    }
    scale_rotations(ops, mats);
    if ((int)ops.size() > KATE_MAX_SOPS || (int)mats.size() > KATE_MAX_MATS)
        return "pass program too large for the kernel parameter";
    out->nops = (int)ops.size();
    out->nmats = (int)mats.size();
    for (size_t i = 0; i < ops.size(); i++) out->ops[i] = ops[i];
    for (size_t i = 0; i < mats.size(); i++) {
        out->mats[i][0] = mats[i].re;
        out->mats[i][1] = mats[i].im;
    }
    return "";
}

}  // namespace kate
