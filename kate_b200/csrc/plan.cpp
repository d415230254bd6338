// Group-pass planner. See plan.hpp.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <set>
#include <system_error>
#include <thread>
#include <unordered_map>

namespace kate {

namespace {

constexpr double kPi = 3.1415926535897932384626433;

bool is_diagonal(const std::vector<Cx>& m, int dim) {
    for (int r = 0; r < dim; r++)
        for (int c = 0; c < dim; c++)
            if (r != c && (m[(size_t)r * dim + c].re != 0.0 || m[(size_t)r * dim + c].im != 0.0)) return false;
    return true;
}

std::string classify(const Gate& g, const std::vector<int>& lab2log, int src, std::vector<PGate>& out) {
    std::vector<int> q;
    for (int x : g.qbits) q.push_back(lab2log[x]);
    PGate p;
    p.src = src;
    switch (g.id) {
    case G_H:
        p.kind = OPK_H;
        p.tq = {q[0]};
        break;
    case G_CNOT:
        p.kind = OPK_X;
        p.tq = {q[0]};
        p.fq = {q[1]};
        break;
    case G_TOFFOLI:
        p.kind = OPK_X;
        p.tq = {q[2]};
        p.fq = {q[0], q[1]};
        break;
    case G_CRK: {
        p.kind = OPK_PHASE;
        p.fq = {q[0], q[1]};
        double t = ((double)2 * kPi) / (double)(1ull << g.optarg);
        p.ph_re = std::cos(t);
        p.ph_im = std::sin(t);
        break;
    }
    case G_DENSE: {
        int k = (int)q.size();
        if (k > 5) return "dense gates above 5 qubits are not supported by the device path (fuse with k <= 5)";
        int dim = 1 << k;
        if (is_diagonal(g.dense, dim)) {
            p.kind = OPK_DIAG;
            p.fq = q;
            for (int i = 0; i < dim; i++) p.table.push_back(g.dense[(size_t)i * dim + i]);
        } else {
            p.kind = OPK_DENSE;
            p.tq = q;
            p.table = g.dense;
        }
        break;
    }
    default:
        return "";  // RX / RZ: no arithmetic, as in the reference
    }
    out.push_back(std::move(p));
    return "";
}

// One-qubit chain fusion (the planner's own GateMerger step): an op acting
// on a single qubit q (dense 2x2, diagonal, H) whose previous op touching q
// is also a single-qubit op on q is multiplied into it in FP64. A layer of
// RX then RZ on every qubit becomes one 2x2 per qubit (8 FMAs per amplitude
// instead of two passes over the tile).
bool single_qubit(const PGate& g, int* q) {
    if ((g.kind == OPK_DENSE || g.kind == OPK_H) && g.tq.size() == 1 && g.fq.empty()) {
        *q = g.tq[0];
        return true;
    }
    if (g.kind == OPK_DIAG && g.fq.size() == 1 && g.tq.empty()) {
        *q = g.fq[0];
        return true;
    }
    return false;
}

void matrix_2x2(const PGate& g, Cx m[4]) {
    if (g.kind == OPK_H) {
        const double s = 0.7071067811865475;
        m[0] = {s, 0};
        m[1] = {s, 0};
        m[2] = {s, 0};
        m[3] = {-s, 0};
    } else if (g.kind == OPK_DIAG) {
        m[0] = g.table[0];
        m[1] = {0, 0};
        m[2] = {0, 0};
        m[3] = g.table[1];
    } else {
        for (int i = 0; i < 4; i++) m[i] = g.table[i];
    }
}

// FP64 operations per amplitude of a 2x2 in the tile kernel (diagonals ~1:
// they merge into the stage's register diagonal).
int cost_2x2(const Cx m[4]) {
    if (m[1].re == 0.0 && m[1].im == 0.0 && m[2].re == 0.0 && m[2].im == 0.0) return 1;
    int k = classify_2x2(m);
    if (k == SOP_U) return 8;
    // Real or RX-form: 2 when a factor can be taken out (a = d, or c = +-b).
    const double a = m[0].re, d = m[3].re;
    const double b = k == SOP_UX ? m[1].im : m[1].re, c = k == SOP_UX ? m[2].im : m[2].re;
    const bool scalable = (a == d && a != 0.0) || (b != 0.0 && (k == SOP_UX ? c == b : c == -b));
    return scalable ? 2 : 4;
}

PGate make_1q(int q, const Cx m[4], int src) {
    PGate p;
    p.src = src;
    if (m[1].re == 0.0 && m[1].im == 0.0 && m[2].re == 0.0 && m[2].im == 0.0) {
        p.kind = OPK_DIAG;
        p.fq = {q};
        p.table = {m[0], m[3]};
    } else {
        p.kind = OPK_DENSE;
        p.tq = {q};
        p.table.assign(m, m + 4);
    }
    return p;
}

std::vector<PGate> fuse_single_qubit(std::vector<PGate>&& in, int n) {
    std::vector<PGate> out;
    out.reserve(in.size());
    std::vector<int> last(n, -1);
    for (auto& g : in) {
        int q;
        if (single_qubit(g, &q) && last[q] >= 0) {
            int q2;
            PGate& prev = out[last[q]];
            if (single_qubit(prev, &q2) && q2 == q) {
                Cx a[4], b[4], r[4];
                matrix_2x2(g, a);
                matrix_2x2(prev, b);
                for (int i = 0; i < 2; i++)
                    for (int j = 0; j < 2; j++) r[2 * i + j] = a[2 * i] * b[j] + a[2 * i + 1] * b[2 + j];
                // Multiply only when the product is no dearer than the two
                // ops apart: diagonals are nearly free (the tile kernel merges
                // all register-bit diagonals of a stage into one multiply),
                // real and RX-form 2x2s cost half a general one.
                if (cost_2x2(r) <= cost_2x2(a) + cost_2x2(b)) {
                    prev = make_1q(q, r, prev.src);
                    continue;
                }
            }
        }
        out.push_back(std::move(g));
        for (int x : out.back().tq) last[x] = (int)out.size() - 1;
        for (int x : out.back().fq) last[x] = (int)out.size() - 1;
    }
    return out;
}

struct Layout {
    std::vector<int> phys;  // logical -> physical
    std::vector<int> inv;   // physical -> logical
    explicit Layout(int n) : phys(n), inv(n) {
        std::iota(phys.begin(), phys.end(), 0);
        std::iota(inv.begin(), inv.end(), 0);
    }
};

// Greedy tile selection over `rem`: returns executed gate indices; `T` is
// extended in place. If `order` is non-null it records the order in which
// qubits joined T.
std::vector<int> greedy_pass(const std::vector<PGate>& pg, const std::vector<int>& rem, int n, int m,
                             std::vector<char>& inT, int& tsize, std::vector<int>* order, size_t scan_limit,
                             bool all_targets = false) {
    std::vector<char> blocked(n, 0);
    std::vector<int> exec;
    size_t scanned = 0;
    int nblocked = 0;
    for (int gi : rem) {
        if (++scanned > scan_limit || nblocked == n) break;
        const PGate& g = pg[gi];
        bool blk = false;
        for (int q : g.tq) blk |= blocked[q] != 0;
        for (int q : g.fq) blk |= blocked[q] != 0;
        if (!blk) {
            // Targets must be tile qubits; so must every qubit when
            // all_targets is set (complex64 blocks).
            int need = 0;
            for (int q : g.tq) need += !inT[q];
            if (all_targets)
                for (int q : g.fq) need += !inT[q];
            if (tsize + need <= m) {
                auto take = [&](int q) {
                    if (!inT[q]) {
                        inT[q] = 1;
                        tsize++;
                        if (order) order->push_back(q);
                    }
                };
                for (int q : g.tq) take(q);
                if (all_targets)
                    for (int q : g.fq) take(q);
                exec.push_back(gi);
                continue;
            }
        }
        for (int q : g.tq) nblocked += !blocked[q], blocked[q] = 1;
        for (int q : g.fq) nblocked += !blocked[q], blocked[q] = 1;
    }
    return exec;
}

// ---- complex64 passes: tensor-core blocks ----
// A complex64 pass applies at most KATE_C64_MAX_BLOCKS dense blocks of at
// most five qubits, all inside one m-qubit tile, each block the product of a
// set of gates. The selector builds the pass block by block: for every gate
// that is ready (all earlier gates on its qubits taken), it grows a qubit set
// from the gate's qubits, up to five, one ready gate's qubits at a time,
// keeping the growth that lets the set absorb the most gates; the set that
// absorbs the most gates overall becomes the next block. A set absorbs every
// remaining gate inside it whose earlier gates (on any of its qubits) are
// taken, so on a brickwork a block holds a light cone of about 5.5 gates
// instead of the 3.7 of a program-order prefix (32-qubit SU(4) brickwork,
// 20 layers: 27 passes of 53 blocks against 42 passes of 83).

// Gates of `live` (program order) that lie inside Q and follow only gates
// already taken: one scan, which stops once every qubit of Q is blocked.
int absorb_set(const std::vector<uint64_t>& gm, const std::vector<int>& live, uint64_t Q, std::vector<int>* out,
               size_t scan_limit) {
    uint64_t blocked = 0;
    int cnt = 0;
    size_t scanned = 0;
    for (int gi : live) {
        if (++scanned > scan_limit) break;
        const uint64_t q = gm[gi];
        if (!(q & ~Q) && !(q & blocked)) {
            cnt++;
            if (out) out->push_back(gi);
        } else {
            blocked |= q;
            if ((blocked & Q) == Q) break;
        }
    }
    return cnt;
}

// Ready gates of `live` once the gates marked in `skip` are taken.
void ready_gates(const std::vector<uint64_t>& gm, const std::vector<int>& live, const std::vector<char>& skip,
                 uint64_t all, size_t scan_limit, std::vector<int>& out) {
    out.clear();
    uint64_t blocked = 0;
    size_t scanned = 0;
    for (int gi : live) {
        if (skip[gi]) continue;
        if (++scanned > scan_limit || blocked == all) break;
        const uint64_t q = gm[gi];
        if (!(q & blocked)) out.push_back(gi);
        blocked |= q;
    }
}

// One complex64 pass: the gates of up to `maxb` blocks, block by block (a
// valid execution order), drawn from `rem` (program order). `inT`/`tsize`
// hold the tile qubits required already (the low physical bits) and receive
// the blocks' qubits; `order` (optional) records qubits as they join.
std::vector<int> c64_pass(const std::vector<PGate>& pg, const std::vector<int>& rem, int n, int m, int maxb,
                          std::vector<char>& inT, int& tsize, std::vector<int>* order, size_t scan_limit) {
    std::vector<uint64_t> gm(pg.size(), 0);
    for (int gi : rem) {
        uint64_t q = 0;
        for (int x : pg[gi].tq) q |= 1ull << x;
        for (int x : pg[gi].fq) q |= 1ull << x;
        gm[gi] = q;
    }
    const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1);
    uint64_t T = 0;
    for (int q = 0; q < n; q++)
        if (inT[q]) T |= 1ull << q;
    std::vector<int> live(rem), exec, ready, seeds, tmp;
    std::vector<char> mark(pg.size(), 0);
    // Absorbed-gate counts by qubit set, for the current `live` (many seeds
    // and growth steps reach the same sets).
    std::unordered_map<uint64_t, int> memo;
    auto count = [&](uint64_t Q) {
        auto it = memo.find(Q);
        if (it != memo.end()) return it->second;
        const int c = absorb_set(gm, live, Q, nullptr, scan_limit);
        memo.emplace(Q, c);
        return c;
    };
    for (int b = 0; b < maxb && !live.empty(); b++) {
        std::fill(mark.begin(), mark.end(), 0);
        memo.clear();
        ready_gates(gm, live, mark, all, scan_limit, seeds);
        int best_cnt = 0, best_tile = 0;
        uint64_t best_Q = 0;
        for (int s : seeds) {
            uint64_t Q = gm[s];
            if (__builtin_popcountll(Q) > 5 || __builtin_popcountll(T | Q) > m) continue;
            tmp.clear();
            int cnt = absorb_set(gm, live, Q, &tmp, scan_limit);
            while (__builtin_popcountll(Q) < 5) {
                for (int gi : tmp) mark[gi] = 1;
                ready_gates(gm, live, mark, all, scan_limit, ready);
                for (int gi : tmp) mark[gi] = 0;
                int gc = cnt, gsize = 0;
                uint64_t gQ = 0;
                for (int gi : ready) {
                    const uint64_t nQ = Q | gm[gi];
                    const int sz = __builtin_popcountll(nQ);
                    if (nQ == Q || sz > 5 || __builtin_popcountll(T | nQ) > m) continue;
                    const int c2 = count(nQ);
                    if (c2 > gc || (c2 == gc && gQ && sz < gsize)) {
                        gc = c2;
                        gQ = nQ;
                        gsize = sz;
                    }
                }
                if (!gQ) break;
                Q = gQ;
                tmp.clear();
                cnt = absorb_set(gm, live, Q, &tmp, scan_limit);
            }
            const int tile = __builtin_popcountll(T | Q);
            if (cnt > best_cnt || (cnt == best_cnt && tile < best_tile)) {
                best_cnt = cnt;
                best_Q = Q;
                best_tile = tile;
            }
        }
        if (best_cnt == 0) break;
        tmp.clear();
        absorb_set(gm, live, best_Q, &tmp, scan_limit);
        for (int gi : tmp) mark[gi] = 1;
        exec.insert(exec.end(), tmp.begin(), tmp.end());
        for (int q = 0; q < n; q++)
            if (((best_Q >> q) & 1ull) && !inT[q]) {
                inT[q] = 1;
                tsize++;
                if (order) order->push_back(q);
            }
        T |= best_Q;
        std::vector<int> nl;
        nl.reserve(live.size());
        for (int gi : live)
            if (!mark[gi]) nl.push_back(gi);
        live.swap(nl);
    }
    return exec;
}

}  // namespace

namespace {

// Evaluates f on every candidate on the calling thread and a few workers
// (kept for one plan); out[k] = f(cands[k]).
class CandPool {
  public:
    explicit CandPool(int workers) : workers_(0) {
        for (int i = 0; i < workers; i++) {
            try {
                th_.emplace_back([this] { loop(); });
                workers_++;
            } catch (const std::system_error&) {
                break;  // fewer workers; the calling thread counts the rest
            }
        }
    }
    ~CandPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    template <typename F>
    void run(const std::vector<uint64_t>& cands, F& f, std::vector<size_t>& out) {
        out.assign(cands.size(), 0);
        if (workers_ == 0) {
            for (size_t k = 0; k < cands.size(); k++) out[k] = f(cands[k]);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            cands_ = &cands;
            out_ = &out;
            fn_ = [&f](uint64_t x) { return f(x); };
            next_ = 0;
            pending_ = workers_;
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    void work() {
        for (size_t k; (k = next_.fetch_add(1)) < cands_->size();) (*out_)[k] = fn_((*cands_)[k]);
    }
    void loop() {
        int seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    int workers_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::vector<uint64_t>* cands_ = nullptr;
    std::vector<size_t>* out_ = nullptr;
    std::function<size_t(uint64_t)> fn_;
    std::atomic<size_t> next_{0};
    int gen_ = 0, pending_ = 0;
    bool stop_ = false;
};

// Workers per plan for the remap search: the four cap plans run at once, so
// a quarter of the host's threads each, the plan's own thread included.
int search_workers() {
    const int hw = (int)std::thread::hardware_concurrency();
    return std::max(0, std::min(3, hw / 4 - 1));
}

}  // namespace

DevPass to_devpass(int n, const PlannedPass& p, int op0) {
    DevPass d{};
    int m = (int)p.phys_in.size();
    d.m = m;
    d.nops = (int)p.ops.size();
    d.op0 = op0;
    d.ncb = n - m;
    std::vector<char> inS(n, 0);
    for (int t = 0; t < m; t++) {
        d.tphys[t] = (uint8_t)p.phys_in[t];
        inS[p.phys_in[t]] = 1;
    }
    for (int t = 0; t < m; t++) d.outsrc[p.out_tile[t]] = (uint8_t)t;
    int j = 0;
    for (int b = 0; b < n; b++)
        if (!inS[b]) d.cphys[j++] = (uint8_t)b;
    return d;
}

void lower_pass(const Plan& plan, PlannedPass& pass, const std::vector<int>& phys, std::vector<Cx>& pool) {
    const int m = (int)pass.phys_in.size();
    auto tile_bit = [&](int q) -> int {
        int p = phys[q];
        for (int t = 0; t < m; t++)
            if (pass.phys_in[t] == p) return t;
        return -1;
    };
    pass.ops.clear();
    for (int gi : pass.gates) {
        const PGate& g = plan.pgates[gi];
        DevOp op{};
        op.kind = g.kind;
        op.k = (int)std::max(g.tq.size(), g.fq.size());
        for (int i = 0; i < 5; i++) op.tb[i] = op.ftb[i] = op.fpos[i] = -1;
        for (size_t i = 0; i < g.tq.size(); i++) op.tb[i] = tile_bit(g.tq[i]);
        op.ph_re = g.ph_re;
        op.ph_im = g.ph_im;
        op.mat = -1;
        if (g.kind == OPK_DENSE) op.k = (int)g.tq.size();
        if (g.kind == OPK_X || g.kind == OPK_PHASE) {
            for (int q : g.fq) {
                int t = tile_bit(q);
                if (t >= 0) op.tmask |= 1u << t;
                else op.pmask |= 1ull << phys[q];
            }
        }
        if (g.kind == OPK_DIAG) {
            op.k = (int)g.fq.size();
            for (size_t i = 0; i < g.fq.size(); i++) {
                int t = tile_bit(g.fq[i]);
                op.ftb[i] = t;
                op.fpos[i] = t >= 0 ? -1 : phys[g.fq[i]];
            }
        }
        if (!g.table.empty()) {
            op.mat = (int64_t)pool.size();
            pool.insert(pool.end(), g.table.begin(), g.table.end());
        }
        pass.ops.push_back(op);
    }
}

std::vector<PlannedPass> plan_relayout(int n, const std::vector<int>& phys0, const std::vector<int>& target,
                                       const PlanOptions& opt) {
    std::vector<PlannedPass> out;
    const int m = std::min(opt.max_tile, n);
    const int c = std::min(opt.coalesce, m);
    std::vector<int> phys(phys0), inv(n);
    for (int q = 0; q < n; q++) inv[phys[q]] = q;
    for (int guard = 0; guard < 4 * n + 8 && phys != target; guard++) {
        std::vector<char> inS(n, 0);
        std::vector<int> S;
        auto add = [&](int p) {
            if (!inS[p] && (int)S.size() < m) {
                inS[p] = 1;
                S.push_back(p);
            }
        };
        for (int p = 0; p < c; p++) add(p);
        // Follow displacement cycles from each wrong position while room remains.
        for (int p = 0; p < n && (int)S.size() < m; p++) {
            if (target[inv[p]] == p) continue;
            int cur = p;
            while ((int)S.size() < m) {
                add(cur);
                int nxt = target[inv[cur]];
                if (inS[nxt]) break;
                cur = nxt;
            }
        }
        for (int p = 0; p < n && (int)S.size() < m; p++) add(p);
        std::sort(S.begin(), S.end());
        // Inside S: every qubit whose target lies in S goes there; the rest
        // fill the remaining positions in order.
        std::vector<int> newpos(n, -1);
        std::vector<char> taken(n, 0);
        for (int p : S) {
            int q = inv[p];
            if (inS[target[q]]) {
                newpos[q] = target[q];
                taken[target[q]] = 1;
            }
        }
        size_t fill = 0;
        for (int p : S) {
            int q = inv[p];
            if (newpos[q] >= 0) continue;
            while (taken[S[fill]]) fill++;
            newpos[q] = S[fill];
            taken[S[fill]] = 1;
        }
        PlannedPass pp;
        pp.phys_in = S;
        pp.out_tile.assign(m, 0);
        for (int t = 0; t < m; t++) {
            int q = inv[S[t]];
            pp.tile.push_back(q);
            int np = newpos[q];
            pp.out_tile[t] = (int)(std::lower_bound(S.begin(), S.end(), np) - S.begin());
        }
        for (int p : S) {
            int q = inv[p];
            phys[q] = newpos[q];
        }
        for (int q = 0; q < n; q++) inv[phys[q]] = q;
        out.push_back(std::move(pp));
    }
    return out;
}

std::string build_plan(const Program& prog, const PlanOptions& opt, Plan* out) {
    if (opt.cap_search && !opt.c64) {
        // One plan per cap, on its own thread.
        const int caps[4] = {96, 112, 128, 144};
        Plan plans[4];
        std::string errs[4];
        auto one = [&](int k) {
            try {
                PlanOptions o = opt;
                o.cap_search = false;
                o.max_gates_per_pass = caps[k];
                errs[k] = build_plan(prog, o, &plans[k]);
            } catch (const std::exception& e) {
                errs[k] = std::string("planner: ") + e.what();
            }
        };
        std::vector<std::thread> th;
        for (int k = 0; k < 4; k++) {
            try {
                th.emplace_back(one, k);
            } catch (const std::system_error&) {
                one(k);  // no thread to spare: plan this cap here
            }
        }
        for (auto& t : th) t.join();
        // Estimated time per amplitude (B200 rates, ps): a pass is bound by
        // HBM (32 B at 6.5 TB/s), FP64 issue (64 per SM-clock, 148 SMs,
        // 1.9 GHz) or its shared-memory exchanges (32 B per amplitude each,
        // 128 B per SM-clock); the on-chip terms carry the 1.5x that the
        // heavy passes measure against them. Passes with shared-memory ops
        // (interpreter) or without a register-staged program (generic
        // kernel) count three and ten HBM passes.
        auto cost = [](const PlannedPass& pp) {
            const double hbm = 4.92;
            if (!pp.prog) return 10 * hbm;
            double f = 0;
            int ex = -1;
            for (int k = 0; k < pp.prog->nops; k++) {
                const SOp& o = pp.prog->ops[k];
                if (o.kind == SOP_SMEM) return 3 * hbm;
                if (o.kind == SOP_STAGE) ex++;
                f += sop_fp64_per_amp(o);
            }
            return std::max(hbm, 1.5 * std::max(0.0556 * f, 0.89 * std::max(ex, 0)));
        };
        double best = -1;
        int bk = -1;
        for (int k = 0; k < 4; k++) {
            if (!errs[k].empty()) continue;
            double score = 0;
            for (const auto& pp : plans[k].passes) score += cost(pp);
            if (best < 0 || score < best) best = score, bk = k;
        }
        if (bk < 0) return errs[0];
        *out = std::move(plans[bk]);
        return "";
    }
    Plan& plan = *out;
    const int n = prog.nqbits;
    plan = Plan();
    plan.n = n;
    plan.dense2_reg = opt.dense2_reg && !opt.c64;
    plan.initial_permutation = prog.initial_permutation;
    plan.final_inverse_permutation = prog.final_inverse_permutation;
    std::vector<int> lab2log(n);
    std::iota(lab2log.begin(), lab2log.end(), 0);
    // Walk the instruction stream: swaps relabel, computes emit gates.
    size_t gi = 0;
    int k = 0;
    for (auto& ins : prog.instructions) {
        if (ins.first == 0) {
            for (size_t i = 0; i + 1 < ins.second.size(); i += 2) {
                int a = ins.second[i], b = ins.second[i + 1];
                if (a < 0 || b < 0 || a >= n || b >= n) return "swap instruction outside the circuit";
                std::swap(lab2log[a], lab2log[b]);
            }
        } else {
            if (gi >= prog.groups.size()) return "instruction stream has more compute steps than groups";
            int end = prog.groups[gi].first;
            for (; k < end; k++) {
                std::string e = classify(prog.gates[k], lab2log, k, plan.pgates);
                if (!e.empty()) return e;
            }
            gi++;
        }
    }
    plan.label_to_logical = lab2log;
    if (opt.fuse_1q) plan.pgates = fuse_single_qubit(std::move(plan.pgates), n);

    const int m = std::min(opt.max_tile, n);
    // Gates of one pass span at most mg qubits (the c low bits included);
    // the tile is then filled up to m with other qubits.
    const int mg = opt.group_qubits > 0 ? std::min(opt.group_qubits, m) : m;
    int maxT = 0;
    for (auto& g : plan.pgates) maxT = std::max(maxT, (int)(g.tq.size() + (opt.c64 ? g.fq.size() : 0)));
    if (maxT > mg) return "a gate has more target qubits than the tile";
    // The c low physical bits are always tile bits; leave room for the
    // widest gate's targets beside them so every pass can make progress.
    const int c = std::max(0, std::min(opt.coalesce, mg - maxT));
    Layout L(n);
    std::vector<int> rem(plan.pgates.size());
    std::iota(rem.begin(), rem.end(), 0);
    const size_t scan_limit = 1u << 20;
    const size_t c64_scan_limit = 1u << 13;  // the block selector scans this window of the remaining gates
    std::vector<uint64_t> qmask, tmask;      // per gate: its qubits, its tile qubits (remap search)
    std::unique_ptr<CandPool> pool;          // threads that count the remap search's candidates
    while (!rem.empty()) {
      // A pass whose register-staged program would not fit (too many
      // matrices or stages) is planned again with three quarters of its
      // gates rather than left to the slower shared-memory ops.
      const std::vector<int> rem0 = rem;
      const size_t pool0 = plan.pool.size(), smem0 = plan.smem_ops.size();
      size_t cap = (size_t)opt.max_gates_per_pass;
      for (;;) {
        std::vector<char> inT(n, 0);
        int tsize = 0;
        for (int p = 0; p < c; p++) {
            inT[L.inv[p]] = 1;
            tsize++;
        }
        const bool blocks = opt.c64 && m == KATE_TILE_BITS;
        std::vector<int> exec = blocks ? c64_pass(plan.pgates, rem, n, mg, KATE_C64_MAX_BLOCKS, inT, tsize, nullptr,
                                                  c64_scan_limit)
                                       : greedy_pass(plan.pgates, rem, n, mg, inT, tsize, nullptr, scan_limit, opt.c64);
        size_t keep = exec.size();
        if (!blocks && keep > cap) keep = cap;
        if (keep < exec.size()) {
            // Keep a prefix of the executable gates (a prefix of a
            // dependency-closed set in program order is dependency-closed).
            exec.resize(keep);
            std::fill(inT.begin(), inT.end(), 0);
            tsize = 0;
            for (int p = 0; p < c; p++) {
                inT[L.inv[p]] = 1;
                tsize++;
            }
            for (int gi : exec) {
                for (int q : plan.pgates[gi].tq)
                    if (!inT[q]) {
                        inT[q] = 1;
                        tsize++;
                    }
                if (opt.c64)
                    for (int q : plan.pgates[gi].fq)
                        if (!inT[q]) {
                            inT[q] = 1;
                            tsize++;
                        }
            }
        }
        if (exec.empty()) return "planner made no progress";
        for (int p = 0; p < n && tsize < m; p++)
            if (!inT[L.inv[p]]) {
                inT[L.inv[p]] = 1;
                tsize++;
            }
        {
            // exec is in block order for complex64 passes, so remove by mark.
            std::vector<char> taken(plan.pgates.size(), 0);
            for (int g : exec) taken[g] = 1;
            std::vector<int> nr;
            nr.reserve(rem.size());
            for (int g : rem)
                if (!taken[g]) nr.push_back(g);
            rem.swap(nr);
        }
        // Tile bits in ascending physical order.
        std::vector<int> S;
        for (int q = 0; q < n; q++)
            if (inT[q]) S.push_back(L.phys[q]);
        std::sort(S.begin(), S.end());
        // Choose the qubits that the next pass wants at the low positions.
        std::vector<int> newlow;
        if (opt.remap && opt.remap_search && !rem.empty() && !blocks && c > 0 && c < m && n <= 64) {
            // Every c-subset of the tile (ascending logical ids, first best
            // kept): the one with which the next pass's greedy selection
            // takes the most gates.
            // The count is greedy_pass's on qubit bitmasks (n <= 64).
            std::vector<int> T;
            for (int q = 0; q < n; q++)
                if (inT[q]) T.push_back(q);
            if (qmask.empty()) {
                qmask.resize(plan.pgates.size());
                tmask.resize(plan.pgates.size());
                for (size_t g = 0; g < plan.pgates.size(); g++) {
                    uint64_t a = 0, t = 0;
                    for (int q : plan.pgates[g].tq) a |= 1ull << q, t |= 1ull << q;
                    for (int q : plan.pgates[g].fq) a |= 1ull << q, t |= opt.c64 ? 1ull << q : 0ull;
                    qmask[g] = a;
                    tmask[g] = t;
                }
            }
            const uint64_t all = n >= 64 ? ~0ull : (1ull << n) - 1;
            auto count = [&](uint64_t low) {
                uint64_t blocked = 0, inT2 = low;
                int ts2 = __builtin_popcountll(low);
                size_t got = 0, scanned = 0;
                for (int gi : rem) {
                    if (blocked == all || ++scanned > scan_limit) break;
                    const uint64_t a = qmask[gi];
                    if (!(a & blocked)) {
                        const uint64_t need = tmask[gi] & ~inT2;
                        const int nn = __builtin_popcountll(need);
                        if (ts2 + nn <= mg) {
                            inT2 |= need;
                            ts2 += nn;
                            got++;
                            continue;
                        }
                    }
                    blocked |= a;
                }
                return got;
            };
            std::vector<uint64_t> cands;
            std::vector<int> idx(c);
            std::iota(idx.begin(), idx.end(), 0);
            const int nt = (int)T.size();
            while (true) {
                uint64_t low = 0;
                for (int i : idx) low |= 1ull << T[i];
                cands.push_back(low);
                int i = c - 1;
                while (i >= 0 && idx[i] == nt - c + i) i--;
                if (i < 0) break;
                idx[i]++;
                for (int j = i + 1; j < c; j++) idx[j] = idx[j - 1] + 1;
            }
            std::vector<size_t> got;
            if (!pool) pool.reset(new CandPool(search_workers()));
            pool->run(cands, count, got);
            size_t best = 0;
            for (size_t k = 0; k < cands.size(); k++)
                if (got[k] > best) {
                    best = got[k];
                    newlow.clear();
                    for (int q = 0; q < n; q++)
                        if ((cands[k] >> q) & 1ull) newlow.push_back(q);
                }
        } else if (opt.remap && !rem.empty()) {
            std::vector<char> inT2(n, 0);
            int ts2 = 0;
            std::vector<int> order;
            greedy_pass(plan.pgates, rem, n, mg, inT2, ts2, &order, scan_limit, opt.c64);
            for (int q : order)
                if (inT[q] && (int)newlow.size() < c) newlow.push_back(q);
        }
        for (int p = 0; p < c && (int)newlow.size() < c; p++) {
            int q = L.inv[p];
            if (std::find(newlow.begin(), newlow.end(), q) == newlow.end()) newlow.push_back(q);
        }
        // New layout: newlow qubits already in the low bits stay; arrivals
        // take the freed low positions; displaced low qubits take the
        // arrivals' old positions.
        std::vector<int> nphys(L.phys);
        std::vector<char> isnew(n, 0);
        for (int q : newlow) isnew[q] = 1;
        std::vector<int> freed, leaving;
        for (int p = 0; p < c; p++)
            if (!isnew[L.inv[p]]) {
                freed.push_back(p);
                leaving.push_back(L.inv[p]);
            }
        size_t fi = 0;
        for (int q : newlow)
            if (L.phys[q] >= c) {
                int oldp = L.phys[q];
                nphys[q] = freed[fi];
                nphys[leaving[fi]] = oldp;
                fi++;
            }
        PlannedPass pp;
        pp.phys_in = S;
        pp.gates = exec;
        pp.out_tile.assign(m, 0);
        for (int t = 0; t < m; t++) {
            int q = L.inv[S[t]];
            pp.tile.push_back(q);
            pp.out_tile[t] = (int)(std::lower_bound(S.begin(), S.end(), nphys[q]) - S.begin());
        }
        lower_pass(plan, pp, L.phys, plan.pool);
        pp.phys_before = L.phys;
        if (opt.c64) {
            if (m == KATE_TILE_BITS) {
                auto bp = std::make_shared<BlockProg>();
                pp.prog_note = build_block_program(plan, pp, n, plan.bimg, bp.get());
                if (pp.prog_note.empty()) pp.bprog = bp;
                else return "complex64 block lowering failed: " + pp.prog_note;
            }
        } else if (opt.staged) {
            auto prog = std::make_shared<PassProg>();
            // Dense two-qubit gates as register ops when asked for; a pass
            // whose program would then not fit the kernel parameter keeps
            // them as shared-memory ops.
            const size_t so = plan.smem_ops.size(), po = plan.pool.size();
            pp.prog_note = opt.dense2_reg ? build_pass_program(plan, pp, n, plan.smem_ops, plan.pool, prog.get(), true)
                                          : std::string("off");
            if (!pp.prog_note.empty() && opt.dense2_reg && exec.size() > 8 &&
                (pp.prog_note.find("too large") != std::string::npos ||
                 pp.prog_note.find("too many") != std::string::npos)) {
                rem = rem0;
                plan.pool.resize(pool0);
                plan.smem_ops.resize(smem0);
                cap = exec.size() * 3 / 4;
                continue;
            }
            if (!pp.prog_note.empty()) {
                plan.smem_ops.resize(so);
                plan.pool.resize(po);
                pp.prog_note = build_pass_program(plan, pp, n, plan.smem_ops, plan.pool, prog.get(), false);
            }
            if (pp.prog_note.empty() && opt.dense2_reg && opt.remap_search) {
                // A first stage that keeps tile bits 0..3 out of its registers
                // loads straight from HBM; kept when the program then needs
                // fewer shared-memory round trips.
                bool low_reg = false;
                for (int i = 0; i < 4; i++) low_reg |= prog->nstages > 0 && prog->srb[0][i] < 4;
                if (low_reg) {
                    std::vector<DevOp> smem_alt(plan.smem_ops.begin(), plan.smem_ops.begin() + (long)so);
                    std::vector<Cx> pool_alt(plan.pool.begin(), plan.pool.begin() + (long)po);
                    auto alt = std::make_shared<PassProg>();
                    const std::string e2 =
                        build_pass_program(plan, pp, n, smem_alt, pool_alt, alt.get(), true, true);
                    if (e2.empty() && prog_round_trips(*alt) < prog_round_trips(*prog)) {
                        plan.smem_ops.swap(smem_alt);
                        plan.pool.swap(pool_alt);
                        prog = alt;
                    }
                }
            }
            if (pp.prog_note.empty()) pp.prog = prog;
        }
        plan.passes.push_back(std::move(pp));
        L.phys = nphys;
        for (int q = 0; q < n; q++) L.inv[L.phys[q]] = q;
        break;
      }
    }
    plan.final_phys = L.phys;
    return "";
}

}  // namespace kate
