// Host compile passes and the FP64 gate merger. See circuit.hpp.
#include "circuit.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <functional>
#include <list>
#include <queue>
#include <set>
#include <unordered_set>

namespace kate {

namespace {

constexpr double kPi = 3.1415926535897932384626433;
constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kSqrt2Inv = 0.7071067811865475;

// Sparse forward DAG with the reference's shortest-path rule
// (backendagnosticcode/graphUtil.hpp:38-80): a binary heap of (dist, node)
// popped smallest-first (ties to the smaller node), neighbours relaxed in
// ascending node order, first reach always accepted, later reaches only when
// strictly shorter, stop when the target is popped. Reproducing this rule
// (not just "a shortest path") keeps tie-breaking, and so the chosen fusion
// intervals and groups, identical to the reference.
struct PathGraph {
    int n;
    std::vector<std::vector<std::pair<int, double>>> adj;  // per node, ascending target
    explicit PathGraph(int n_) : n(n_), adj(n_) {}
    void edge(int i, int j, double w) { adj[i].emplace_back(j, w); }
    std::vector<int> path(int src, int dst) {
        for (auto& a : adj) std::sort(a.begin(), a.end(), [](auto& x, auto& y) { return x.first < y.first; });
        using QE = std::pair<double, int>;
        std::priority_queue<QE, std::vector<QE>, std::greater<QE>> q;
        std::vector<double> dist(n, 0.0);
        std::vector<int> pred(n, -1);
        dist[src] = 0;
        pred[src] = -2;
        q.push({0.0, src});
        while (!q.empty()) {
            int u = q.top().second;
            q.pop();
            if (u == dst) break;
            for (auto& [k, p] : adj[u]) {
                if (pred[k] == -1) {
                    pred[k] = u;
                    dist[k] = dist[u] + p;
                    q.push({dist[k], k});
                } else if (dist[k] > dist[u] + p) {
                    pred[k] = u;
                    dist[k] = dist[u] + p;
                    q.push({dist[k], k});
                }
            }
        }
        if (pred[dst] == -1) return {-1};
        std::vector<int> r;
        for (int v = dst; v != -2; v = pred[v]) r.push_back(v);
        std::reverse(r.begin(), r.end());
        return r;
    }
};

std::vector<int> sorted_unique(const std::vector<int>& v) {
    std::vector<int> s(v);
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
    return s;
}

}  // namespace

std::string validate_gate(const Program& p, const Gate& g) {
    int nq = (int)g.qbits.size();
    for (int q : g.qbits)
        if (q < 0 || q >= p.nqbits) return "gate qubit " + std::to_string(q) + " outside the circuit's " +
                                             std::to_string(p.nqbits) + " qubits";
    for (int i = 0; i < nq; i++)
        for (int j = i + 1; j < nq; j++)
            if (g.qbits[i] == g.qbits[j]) return "a qubit is present twice in the gate: " + std::to_string(g.qbits[i]);
    switch (g.id) {
    case G_DENSE:
        if (nq < 1 || nq > 10) return "dense gates take 1 to 10 qubits";
        if (g.dense.size() != ((size_t)1 << (2 * nq))) return "dense matrix dimension does not match 2^k";
        break;
    case G_H: if (nq != 1) return "hadamard is on exactly 1 qubit"; break;
    case G_CNOT: if (nq != 2) return "CNOT is on exactly 2 qubits"; break;
    case G_CRK:
        if (nq != 2) return "controlled Rk is on exactly 2 qubits";
        if (g.optarg < 0 || g.optarg > 62) return "CRk's k must be in [0, 62]";
        break;
    case G_TOFFOLI: if (nq != 3) return "toffoli is on exactly 3 qubits"; break;
    case G_RX:
    case G_RZ: if (nq != 1) return "RX/RZ are on exactly 1 qubit"; break;
    default: return "unknown gate identifier " + std::to_string(g.id);
    }
    if (!p.groups.empty()) return "gates cannot be appended after gateGrouping/allocate";
    return "";
}

// Local-state gate application with the reference's arithmetic
// (CPUcode/GateComputing.hpp:6-129). local_bits[i] is the local bit of
// g.qbits[i].
void apply_gate_local(const Gate& g, const int* lb, int k, Cx* st) {
    const int nq = (int)g.qbits.size();
    int sorted[16];
    std::copy(lb, lb + nq, sorted);
    std::sort(sorted, sorted + nq);
    auto ins = [&](uint64_t line, int cnt) {
        uint64_t v = line;
        for (int i = 0; i < cnt; i++) {
            uint64_t p = (uint64_t)sorted[i];
            v = ((v >> p) << (p + 1)) | (v & ((1ull << p) - 1));
        }
        return v;
    };
    switch (g.id) {
    case G_TOFFOLI:
        for (uint64_t line = 0; line < (1ull << (k - 3)); line++) {
            uint64_t a = ins(line, 3) + (1ull << lb[0]) + (1ull << lb[1]);
            uint64_t b = a + (1ull << lb[2]);
            std::swap(st[a], st[b]);
        }
        break;
    case G_CRK: {
        for (uint64_t line = 0; line < (1ull << (k - 2)); line++) {
            uint64_t a = ins(line, 2) + (1ull << lb[1]) + (1ull << lb[0]);
            double t = ((double)2 * kPi) / (double)(1ull << g.optarg);
            Cx ph(std::cos(t), std::sin(t));
            double tr = st[a].re;
            st[a].re = st[a].re * ph.re - st[a].im * ph.im;
            st[a].im = tr * ph.im + st[a].im * ph.re;
        }
        break;
    }
    case G_CNOT:
        for (uint64_t line = 0; line < (1ull << (k - 2)); line++) {
            uint64_t a = ins(line, 2) + (1ull << lb[1]);
            uint64_t b = a + (1ull << lb[0]);
            std::swap(st[a], st[b]);
        }
        break;
    case G_H:
        for (uint64_t line = 0; line < (1ull << (k - 1)); line++) {
            uint64_t a = ins(line, 1);
            uint64_t b = a + (1ull << lb[0]);
            st[a] = (st[a] + st[b]) * kSqrt2Inv;
            st[b] = st[a] - st[b] * kSqrt2;
        }
        break;
    case G_DENSE: {
        const int dim = 1 << nq;
        Cx cache_small[32];
        std::vector<Cx> cache_big(dim > 32 ? dim : 0);
        Cx* cache = dim > 32 ? cache_big.data() : cache_small;
        for (uint64_t line = 0; line < (1ull << (k - nq)); line++) {
            uint64_t base = ins(line, nq);
            for (int s = 0; s < dim; s++) {
                uint64_t idx = base;
                for (int i = 0; i < nq; i++) idx += (uint64_t)((s >> i) & 1) << lb[i];
                cache[s] = st[idx];
            }
            for (int r = 0; r < dim; r++) {
                Cx sum(0.0, 0.0);
                for (int c = 0; c < dim; c++) sum = sum + g.dense[(size_t)r * dim + c] * cache[c];
                uint64_t idx = base;
                for (int i = 0; i < nq; i++) idx += (uint64_t)((r >> i) & 1) << lb[i];
                st[idx] = sum;
            }
        }
        break;
    }
    default:
        break;  // RX/RZ: no arithmetic, as in the reference
    }
}

std::string merge_gates(const std::vector<Gate>& gates, Gate* out) {
    std::vector<int> all;
    for (auto& g : gates) all.insert(all.end(), g.qbits.begin(), g.qbits.end());
    std::vector<int> cov = sorted_unique(all);
    const int k = (int)cov.size();
    if (k > 10) return "merged gate would cover more than 10 qubits";
    const int dim = 1 << k;
    std::vector<Cx> m((size_t)dim * dim);
    for (int r = 0; r < dim; r++)
        for (int c = 0; c < dim; c++) m[(size_t)r * dim + c] = Cx((double)(int)(r == c), 0.0);
    // Local bits of every gate, once (the columns are simulated one by one).
    std::vector<int> lbs;
    std::vector<size_t> lb0;
    for (auto& g : gates) {
        lb0.push_back(lbs.size());
        for (int q : g.qbits) lbs.push_back((int)(std::lower_bound(cov.begin(), cov.end(), q) - cov.begin()));
    }
    for (int col = 0; col < dim; col++)
        for (size_t i = 0; i < gates.size(); i++)
            apply_gate_local(gates[i], lbs.data() + lb0[i], k, m.data() + (size_t)col * dim);
    for (int r = 0; r < dim; r++)
        for (int c = r + 1; c < dim; c++) std::swap(m[(size_t)r * dim + c], m[(size_t)c * dim + r]);
    out->id = G_DENSE;
    out->qbits = cov;
    out->optarg = 0;
    out->dense = std::move(m);
    return "";
}

// gateScheduling (backendagnosticcode/Circuit.hpp:12-98): greedy reverse
// topological order over the ready list, scored against the previous gate's
// qubit set.
//
// The reference computes the score as `qbits.size() - union.size()` in
// size_t, so a gate that adds new qubits scores 2^64 - d (about 1.8e19 as a
// double) and one that adds none scores 0; the running best is an int, and
// storing 1.8e19 into it yields INT_MIN on x86-64 (Circuit.hpp:69-75). The
// effective rule is therefore: the winner is the first no-new-qubit gate
// after the last new-qubit gate, else the last new-qubit gate, else the first
// gate. The loop below reproduces that arithmetic exactly so that schedules
// match the reference's.
std::string pass_schedule(Program& p) {
    const int G = (int)p.gates.size();
    if (G == 0) return "";
    std::vector<std::vector<int>> succ(G), pred(G);
    std::vector<int> lastused(p.nqbits, -1);
    std::unordered_set<uint64_t> seen;
    for (int i = 0; i < G; i++) {
        for (int q : p.gates[i].qbits) {
            if (lastused[q] == -1) {
                lastused[q] = i;
            } else {
                uint64_t key = ((uint64_t)lastused[q] << 32) | (uint32_t)i;
                if (seen.insert(key).second) {
                    succ[lastused[q]].push_back(i);
                    pred[i].push_back(lastused[q]);
                }
                lastused[q] = i;
            }
        }
    }
    std::list<int> ready;
    for (int i = 0; i < G; i++)
        if (succ[i].empty()) ready.push_back(i);
    std::vector<int> remaining(G);
    for (int i = 0; i < G; i++) remaining[i] = (int)succ[i].size();
    std::vector<int> order;
    std::set<int> last;
    while (!ready.empty()) {
        auto best = ready.begin();
        int cur = -INT32_MAX;
        for (auto it = ready.begin(); it != ready.end(); ++it) {
            const auto& qb = p.gates[*it].qbits;
            std::set<int> u(last);
            u.insert(qb.begin(), qb.end());
            double w = (double)((uint64_t)qb.size() - (uint64_t)u.size());
            if (w > (double)cur) {
                cur = (w >= 2147483648.0 || w < -2147483648.0) ? INT_MIN : (int)w;
                best = it;
            }
        }
        int u = *best;
        ready.erase(best);
        order.push_back(u);
        last = std::set<int>(p.gates[u].qbits.begin(), p.gates[u].qbits.end());
        for (int e : pred[u])
            if (--remaining[e] == 0) ready.push_back(e);
    }
    std::vector<Gate> ng;
    ng.reserve(G);
    for (int i = (int)order.size() - 1; i >= 0; i--) ng.push_back(std::move(p.gates[order[i]]));
    p.gates = std::move(ng);
    return "";
}

// gateFusion (backendagnosticcode/Circuit.hpp:99-175): shortest path over
// merge intervals [i, j) with at most `limit` distinct qubits; cost 2^|q|
// per merged block plus merge_time_matters * sum 2^|q_j| * 4^|q| / 2^n, and
// the per-gate costs H 2, CNOT 0.75, CRk 0.25, TOFFOLI 3/8, dense 2^k.
std::string pass_fuse(Program& p, int limit, double mtm, BlockMerger merger, void* ctx) {
    const int G = (int)p.gates.size();
    if (G == 0) return "";
    if (limit > 10) return "fusion is limited to 10-qubit blocks";
    PathGraph graph(G + 1);
    for (int i = 0; i < G; i++) {
        std::set<int> pre(p.gates[i].qbits.begin(), p.gates[i].qbits.end());
        double t;
        switch (p.gates[i].id) {
        case G_DENSE: t = (double)(1ull << pre.size()); graph.edge(i, i + 1, t); break;
        case G_H: graph.edge(i, i + 1, 2.0); break;
        case G_CNOT: graph.edge(i, i + 1, 0.75); break;
        case G_CRK: graph.edge(i, i + 1, 0.25); break;
        case G_TOFFOLI: graph.edge(i, i + 1, (double)3 / 8); break;
        default: break;  // RX/RZ: no single-gate edge, as in the reference
        }
        double t2 = 0;
        for (int j = i + 1; j < G; j++) {
            pre.insert(p.gates[j].qbits.begin(), p.gates[j].qbits.end());
            if ((int)pre.size() > limit) break;
            t2 += (double)(1ull << p.gates[j].qbits.size());
            t = (double)(1ull << pre.size());
            t += mtm * t2 * (double)(1ull << (2 * pre.size())) / (double)(1ull << p.nqbits);
            graph.edge(i, j + 1, t);
        }
    }
    std::vector<int> path = graph.path(0, G);
    if (path.size() == 1 && path[0] == -1)
        return "gateFusion found no merge path (a gate has no cost entry and cannot be merged)";
    std::vector<Gate> out;
    std::vector<std::vector<Gate>> blocks;  // merged intervals, when a block merger is given
    std::vector<size_t> slot;               // their positions in `out`
    int f = -1;
    for (int el : path) {
        if (f == -1) {
            f = el;
            continue;
        }
        if (el == f + 1) {
            out.push_back(p.gates[f]);
        } else {
            std::vector<Gate> block(p.gates.begin() + f, p.gates.begin() + el);
            if (merger) {
                slot.push_back(out.size());
                out.emplace_back();
                blocks.push_back(std::move(block));
            } else {
                Gate m;
                std::string err = merge_gates(block, &m);
                if (!err.empty()) return err;
                out.push_back(std::move(m));
            }
        }
        f = el;
    }
    if (merger && !blocks.empty()) {
        std::vector<Gate> merged;
        std::string err = merger(blocks, ctx, &merged);
        if (!err.empty()) return err;
        if (merged.size() != blocks.size()) return "internal: block merger returned a wrong count";
        for (size_t b = 0; b < slot.size(); b++) out[slot[b]] = std::move(merged[b]);
    }
    p.gates = std::move(out);
    return "";
}

// gateGrouping (backendagnosticcode/Circuit.hpp:176-206): fewest contiguous
// groups with at most `m` distinct qubits, by unit-weight shortest path.
std::string pass_group(Program& p, int m) {
    const int G = (int)p.gates.size();
    if (G == 0) {
        p.groups.clear();
        return "";
    }
    for (auto& g : p.gates)
        if ((int)g.qbits.size() > m) return "a gate has more qubits than the group size";
    PathGraph graph(G + 1);
    for (int i = 0; i < G; i++) {
        std::set<int> pre;
        for (int j = i; j < G; j++) {
            pre.insert(p.gates[j].qbits.begin(), p.gates[j].qbits.end());
            if ((int)pre.size() > m) break;
            graph.edge(i, j + 1, 1.0);
        }
    }
    std::vector<int> fg = graph.path(0, G);
    std::vector<std::pair<int, std::vector<int>>> groups(fg.size() - 1);
    size_t grp = 1;
    std::set<int> pre;
    for (int i = 0; i < G; i++) {
        if (fg[grp] == i) {
            groups[grp - 1] = {i, std::vector<int>(pre.begin(), pre.end())};
            pre.clear();
            grp++;
        }
        pre.insert(p.gates[i].qbits.begin(), p.gates[i].qbits.end());
    }
    groups.back() = {G, std::vector<int>(pre.begin(), pre.end())};
    p.groups = std::move(groups);
    return "";
}

namespace {
void ensure_naive_groups(Program& p) {
    if (!p.groups.empty()) return;
    for (int i = 0; i < (int)p.gates.size(); i++)
        p.groups.push_back({i + 1, sorted_unique(p.gates[i].qbits)});
}

void relabel_group(Program& p, int gi, int& k, const std::vector<int>& perm) {
    std::set<int> t;
    for (int q : p.groups[gi].second) t.insert(perm[q]);
    p.groups[gi].second.assign(t.begin(), t.end());
    for (int l = k; l < p.groups[gi].first; l++)
        for (int& q : p.gates[l].qbits) q = perm[q];
    k = p.groups[gi].first;
}
}  // namespace

// allocate (backendagnosticcode/Circuit.hpp:207-348): Belady-style choice
// of local qubits with swap instructions; with numberofgpulog2 = 0 it emits
// no swap but may relabel qubits by last use.
std::string pass_allocate(Program& p, int g, int maxlocal) {
    const int n = p.nqbits;
    if (maxlocal + g < n) return "cannot allocate: too many qubits for the local qubits and devices";
    if (g < 0 || g >= n) return "numberofgpulog2 out of range";
    maxlocal = n - g;
    p.instructions.clear();
    ensure_naive_groups(p);
    const int NG = (int)p.groups.size();
    std::vector<std::set<std::pair<int, int>>> pre(NG);
    std::vector<int> last_seen(n, INT32_MAX);
    for (int i = NG - 1; i >= 0; i--)
        for (int el : p.groups[i].second) {
            pre[i].insert({el, last_seen[el] - i});
            last_seen[el] = i;
        }
    std::vector<int> ids(n);
    for (int i = 0; i < n; i++) ids[i] = i;
    std::sort(ids.begin(), ids.end(), [&last_seen](int a, int b) { return last_seen[a] < last_seen[b]; });
    std::vector<int> nextsee(last_seen), perm(n), inv(n);
    for (int i = 0; i < n; i++) {
        perm[ids[i]] = i;
        inv[i] = ids[i];
    }
    p.initial_permutation = perm;
    int k = 0;
    for (int i = 0; i < NG; i++) {
        for (int l = 0; l < n; l++) nextsee[l] -= 1;
        std::vector<std::pair<int, int>> pairs;
        std::set<int> taken(p.groups[i].second.begin(), p.groups[i].second.end());
        for (int el : p.groups[i].second) {
            if (perm[el] >= maxlocal) {
                int worst = -1;
                for (int j = 0; j < maxlocal; j++) {
                    if (taken.count(inv[j])) continue;
                    if (worst == -1) {
                        worst = inv[j];
                        continue;
                    }
                    if (nextsee[inv[j]] > nextsee[worst]) worst = inv[j];
                }
                if (worst == -1) return "allocation failed: not enough local qubits for a group";
                pairs.push_back({perm[el], perm[worst]});
                std::swap(inv[perm[el]], inv[perm[worst]]);
                std::swap(perm[el], perm[worst]);
            }
            nextsee[el] = INT32_MAX;
        }
        for (auto& rp : pre[i]) nextsee[rp.first] = rp.second;
        if (!pairs.empty()) {
            std::vector<int> ps;
            for (auto& pr : pairs) {
                ps.push_back(pr.first);
                ps.push_back(pr.second);
            }
            p.instructions.push_back({0, ps});
        }
        p.instructions.push_back({1, {}});
        relabel_group(p, i, k, perm);
    }
    p.final_inverse_permutation = inv;
    return "";
}

// compileDefault (backendagnosticcode/QuantumCircuit.hpp:126-204): one group
// per gate if ungrouped, identity initial permutation, naive swaps.
std::string pass_compile_default(Program& p, int g, int maxlocal) {
    if (!p.instructions.empty()) return "";
    const int n = p.nqbits;
    if (maxlocal + g < n) return "cannot allocate: too many qubits for the local qubits and devices";
    if (g < 0 || g >= n) return "numberofgpulog2 out of range";
    maxlocal = n - g;
    ensure_naive_groups(p);
    std::vector<int> perm(n), inv(n);
    for (int i = 0; i < n; i++) perm[i] = inv[i] = i;
    p.initial_permutation = perm;
    int k = 0;
    for (int gi = 0; gi < (int)p.groups.size(); gi++) {
        std::vector<std::pair<int, int>> pairs;
        std::set<int> taken(p.groups[gi].second.begin(), p.groups[gi].second.end());
        for (int q : p.groups[gi].second) {
            if (perm[q] >= maxlocal) {
                int nl = -1;
                for (int j = 0; j < maxlocal; j++) {
                    if (taken.count(inv[j])) continue;
                    nl = inv[j];
                    break;
                }
                if (nl == -1) return "allocation failed: not enough local qubits for a group";
                pairs.push_back({perm[q], perm[nl]});
                std::swap(inv[perm[q]], inv[perm[nl]]);
                std::swap(perm[q], perm[nl]);
            }
        }
        if (!pairs.empty()) {
            std::vector<int> ps;
            for (auto& pr : pairs) {
                ps.push_back(pr.first);
                ps.push_back(pr.second);
            }
            p.instructions.push_back({0, ps});
        }
        p.instructions.push_back({1, {}});
        relabel_group(p, gi, k, perm);
    }
    p.final_inverse_permutation = inv;
    return "";
}

// exportqcx (backendagnosticcode/Circuit.hpp:763-774 and
// basic_host_types.hpp:270-295): QUBITS n, one line per gate, BEGIN MEASUREMENT.
std::string export_qcx(const Program& p, const std::string& path) {
    std::ofstream f(path);
    if (!f) return "could not open " + path + " to write the qcx file";
    f << "QUBITS " << p.nqbits << "\n";
    for (auto& g : p.gates) {
        std::string s;
        switch (g.id) {
        case G_H: s = "H"; break;
        case G_DENSE: s.assign(g.qbits.size(), 'X'); break;
        case G_CNOT: s = "CNOT"; break;
        case G_CRK: s = "U"; break;
        case G_TOFFOLI: s = "TOFFOLI"; break;
        default: break;
        }
        s += " ";
        for (int q : g.qbits) s += std::to_string(q) + " ";
        if (g.id == G_CRK) s += std::to_string(g.optarg);
        f << s << "\n";
    }
    f << "BEGIN MEASUREMENT";
    return "";
}

}  // namespace kate
