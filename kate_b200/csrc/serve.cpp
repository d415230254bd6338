// Serving engine. See serve.hpp.
#include "serve.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>

#include "devcache.hpp"
#include "launch.hpp"

namespace kate {

namespace {

std::string cuda_err(const char* what, cudaError_t e) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}

// Power-of-two blocks inside [0, total): block sizes min_block << k.
class Buddy {
public:
    void init(uint64_t total, uint64_t min_block, int maxk) {
        min_ = min_block;
        maxk_ = maxk;
        free_.assign(maxk + 1, {});
        uint64_t o = 0;
        while (o + min_ <= total) {
            int k = maxk;
            while (k > 0 && ((o % (min_ << k)) != 0 || o + (min_ << k) > total)) k--;
            free_[k].insert(o);
            o += min_ << k;
        }
    }
    bool alloc(uint64_t bytes, uint64_t* off) {
        int k = 0;
        while ((min_ << k) < bytes) {
            if (++k > maxk_) return false;
        }
        int j = k;
        while (j <= maxk_ && free_[j].empty()) j++;
        if (j > maxk_) return false;
        uint64_t o = *free_[j].begin();
        free_[j].erase(free_[j].begin());
        while (j > k) {
            j--;
            free_[j].insert(o + (min_ << j));
        }
        used_[o] = k;
        *off = o;
        return true;
    }
    void release(uint64_t o) {
        auto it = used_.find(o);
        if (it == used_.end()) return;
        int k = it->second;
        used_.erase(it);
        while (k < maxk_) {
            const uint64_t b = o ^ (min_ << k);
            auto f = free_[k].find(b);
            if (f == free_[k].end()) break;
            free_[k].erase(f);
            o = std::min(o, b);
            k++;
        }
        free_[k].insert(o);
    }

private:
    uint64_t min_ = 1;
    int maxk_ = 0;
    std::vector<std::set<uint64_t>> free_;
    std::unordered_map<uint64_t, int> used_;
};

// First fit over [0, total) in 256-byte units.
class FirstFit {
public:
    void init(uint64_t total) { free_[0] = total; }
    bool alloc(uint64_t bytes, uint64_t* off) {
        bytes = (bytes + 255) & ~uint64_t(255);
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= bytes) {
                *off = it->first;
                const uint64_t rest = it->second - bytes, o2 = it->first + bytes;
                free_.erase(it);
                if (rest) free_[o2] = rest;
                size_[*off] = bytes;
                return true;
            }
        return false;
    }
    void release(uint64_t off) {
        auto s = size_.find(off);
        if (s == size_.end()) return;
        uint64_t o = off, n = s->second;
        size_.erase(s);
        auto next = free_.lower_bound(o);
        if (next != free_.end() && next->first == o + n) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == o) {
                prev->second += n;
                return;
            }
        }
        free_[o] = n;
    }

private:
    std::map<uint64_t, uint64_t> free_;
    std::map<uint64_t, uint64_t> size_;
};

uint64_t splitmix(uint64_t& s) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

struct Req {
    int64_t id = 0;
    Program prog;
    int shots = 0;
    uint64_t seed = 0;
    double t_submit = 0, t_admit = 0;
    bool planned = false;
    CircPack pack;
    std::vector<double> unif;
    // Admission.
    uint64_t state_off = 0, aux_off = 0;
    int64_t prog0 = 0, zoff = 0, poff = 0, uoff = 0, soff = 0;
    uint32_t ncos = 1, nch = 1;
    int npass = 0, levels = 0, next_level = 0;
    BatchCirc circ{};
};

}  // namespace

struct ServerImpl {
    int device = 0, precision = 1;
    ServeOptions opt;
    std::chrono::steady_clock::time_point t0;
    void* d_state = nullptr;
    unsigned char* d_aux = nullptr;
    // Two step slots: while one step runs, the next one is already queued
    // behind it on the stream; results of a finished step are copied on a
    // second stream so they do not wait for the queued step.
    struct Slot {
        BatchTask* d_tasks = nullptr;
        size_t tasks_cap = 0;
        BatchCirc* d_circs = nullptr;
        size_t circs_cap = 0;
        int* d_ctr = nullptr;           // [0] queue head, [1] error flag, [2..] per-circuit done counters
        BatchTask* h_tasks = nullptr;   // pinned
        size_t h_tasks_cap = 0;
        int* h_err = nullptr;           // pinned
        cudaEvent_t ev = nullptr;
        std::vector<Req*> finishing;    // requests whose last level runs in this step
        double t_launch = 0;
    } slots[2];
    int slot_next = 0;
    std::deque<int> inflight;  // launched steps, oldest first
    static constexpr int kMaxStepCircuits = 65536;
    cudaStream_t stream = nullptr;   // uploads and steps
    cudaStream_t cstream = nullptr;  // result copies
    int grid = 0;
    Buddy states;
    FirstFit aux;

    std::mutex m;
    std::condition_variable cv_plan, cv_engine, cv_done;
    bool stop = false;
    int64_t next_id = 0, next_admit = 0;
    std::deque<Req*> planq;
    std::map<int64_t, Req*> waiting;  // submitted, not admitted (planned or not)
    std::vector<Req*> live;
    std::unordered_map<int64_t, ServeResult> results;
    std::unordered_map<int64_t, std::string> failures;
    int64_t n_submitted = 0, n_completed = 0, n_failed = 0, n_steps = 0;
    // Engine thread time, microseconds: admission (plan upload), step task
    // building, step launch to completion, result collection.
    std::atomic<int64_t> us_admit{0}, us_build{0}, us_kernel{0}, us_collect{0};
    std::atomic<uint64_t> resident{0}, peak_resident{0};
    std::vector<std::thread> planners;
    std::thread engine;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    size_t amp_bytes() const { return precision == 0 ? 16 : 8; }

    void plan_loop() {
        for (;;) {
            Req* r;
            {
                std::unique_lock<std::mutex> lk(m);
                cv_plan.wait(lk, [&] { return stop || !planq.empty(); });
                if (stop) return;
                r = planq.front();
                planq.pop_front();
            }
            std::string e;
            try {
                e = pack_circuit(r->prog, opt.tune, true, r->pack, precision == 1);
            } catch (const std::exception& ex) {
                e = ex.what();
            }
            if (e.empty()) {
                uint64_t s = r->seed;
                r->unif.resize(r->shots);
                for (auto& u : r->unif) u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
                std::sort(r->unif.begin(), r->unif.end());
            }
            {
                std::lock_guard<std::mutex> lk(m);
                r->pack.err = e;
                r->planned = true;
            }
            cv_engine.notify_one();
        }
    }

    // Places request r's programs, outputs and uniforms in the aux arena
    // and its state in the state arena. Caller holds no lock.
    bool admit(Req* r) {
        CircPack& P = r->pack;
        const int n = P.n_sim;
        const uint64_t sbytes = (1ull << n) * amp_bytes();
        r->ncos = 1u << (n - KATE_TILE_BITS);
        r->nch = (uint32_t)std::max<uint64_t>(1, (1ull << n) >> 16);
        // Section sizes with worst-case padding for element alignment.
        const uint64_t need = P.progs.size() * sizeof(BatchProg) + P.blob.size() + P.sops.size() * sizeof(DevOp) +
                              P.pool.size() * 16 + 8 * (uint64_t)P.n_out + 8 * (2ull * r->nch + 1) +
                              16 * (uint64_t)r->shots + 8 * 256;
        uint64_t so = 0, ao = 0;
        if (!states.alloc(sbytes, &so)) return false;
        if (!aux.alloc(need, &ao)) {
            states.release(so);
            return false;
        }
        r->state_off = so;
        r->aux_off = ao;
        uint64_t o = ao;
        auto place = [&](uint64_t bytes, uint64_t elem) {
            o = round_up(o, std::max<uint64_t>(elem, 16));
            while (o % elem) o += 16;
            const uint64_t at = o;
            o += bytes;
            return at;
        };
        const uint64_t o_progs = place(P.progs.size() * sizeof(BatchProg), sizeof(BatchProg));
        const uint64_t o_blob = place(P.blob.size(), 16);
        const uint64_t o_sops = place(P.sops.size() * sizeof(DevOp), sizeof(DevOp));
        const uint64_t o_pool = place(P.pool.size() * 16, 16);
        // <Z> and the samples back to back: one copy returns both.
        const uint64_t o_z = place(8 * P.n_out + 8 * (uint64_t)r->shots, 8);
        const uint64_t o_s = o_z + 8 * P.n_out;
        const uint64_t o_ps = place(8 * (2ull * r->nch + 1), 8);
        const uint64_t o_u = place(8 * (uint64_t)r->shots, 8);
        r->prog0 = (int64_t)(o_progs / sizeof(BatchProg));
        r->zoff = (int64_t)(o_z / 8);
        r->poff = (int64_t)(o_ps / 8);
        r->uoff = (int64_t)(o_u / 8);
        r->soff = (int64_t)(o_s / 8);
        // Rebase and upload.
        std::vector<BatchProg> progs = P.progs;
        const int64_t sbase = (int64_t)(o_sops / sizeof(DevOp)), pbase = (int64_t)(o_pool / 16);
        for (auto& bp : progs) {
            bp.ops_off += o_blob;
            bp.mats_off += o_blob;
            bp.stab_off += o_blob;
            bp.sop0 += (int32_t)sbase;
        }
        std::vector<uint8_t> blob = P.blob;
        for (auto& g : P.generic) {
            DevOp* ops = reinterpret_cast<DevOp*>(blob.data() + g.first);
            for (int k = 0; k < g.second; k++) ops[k].mat += pbase;
        }
        std::vector<DevOp> sops = P.sops;
        for (auto& d : sops) d.mat += pbase;
        auto up = [&](uint64_t at, const void* src, size_t bytes) {
            if (bytes) cudaMemcpyAsync(d_aux + at, src, bytes, cudaMemcpyHostToDevice, stream);
        };
        up(o_progs, progs.data(), progs.size() * sizeof(BatchProg));
        up(o_blob, blob.data(), blob.size());
        up(o_sops, sops.data(), sops.size() * sizeof(DevOp));
        up(o_pool, P.pool.data(), P.pool.size() * 16);
        up(o_u, r->unif.data(), r->unif.size() * 8);
        cudaMemsetAsync(d_aux + o_z, 0, 8 * P.n_out, stream);
        r->npass = (int)P.progs.size();
        r->levels = r->npass + 3;  // passes, <Z> + chunk sums, prefix, sampling
        r->next_level = 0;
        BatchCirc& c = r->circ;
        c = BatchCirc{};
        c.off = so / amp_bytes();
        c.n = P.n_out;
        c.shots = r->shots;
        c.zoff = r->zoff;
        c.poff = r->poff;
        c.uoff = r->uoff;
        c.soff = r->soff;
        for (int x = 0; x < P.n_out; x++) c.zbit[x] = P.zbit[x];
        resident += sbytes;
        if (resident.load() > peak_resident.load()) peak_resident = resident.load();
        // The host copies of the plan are no longer needed.
        std::vector<uint8_t>().swap(P.blob);
        std::vector<Cx>().swap(P.pool);
        std::vector<DevOp>().swap(P.sops);
        return true;
    }

    void release(Req* r) {
        states.release(r->state_off);
        aux.release(r->aux_off);
        resident -= (1ull << r->pack.n_sim) * amp_bytes();
    }

    // Estimated latency of level a of r in microseconds (the levels of a
    // request run one after another inside a step): waves of tasks over the
    // CTAs, about 20 us per 4096-amplitude tile pass plus 5 us per task.
    double level_latency_us(const Req* r, int a) const {
        if (a < r->npass) {
            const uint32_t ch = std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)std::max(1, opt.chunk), r->ncos / 64));
            const uint64_t tasks = (r->ncos + ch - 1) / ch;
            const uint64_t waves = (tasks + grid - 1) / std::max(1, grid);
            return (double)waves * (20.0 * ch + 5.0);
        }
        if (a == r->npass) return 5.0 + 2.0 * std::min<uint32_t>(r->nch, (uint32_t)std::max(1, opt.zchunks)) * 8.0;
        if (a == r->npass + 1) return 5.0;
        return 20.0;
    }

    // Cost of level a of r in tile passes (for the step budget).
    int64_t level_cost(const Req* r, int a) const {
        if (a < r->npass) return r->ncos;
        if (a == r->npass) return std::max<int64_t>(1, r->ncos / 2);
        if (a == r->npass + 1) return 1;
        return std::max<int64_t>(1, r->ncos / 4);
    }

    std::string ensure(void** p, size_t* cap, size_t bytes) {
        if (bytes <= *cap) return "";
        if (*p) cudaFree(*p);
        *p = nullptr;
        size_t c = std::max<size_t>(bytes, 2 * *cap);
        cudaError_t e = cudaMalloc(p, c);
        if (e != cudaSuccess) {
            *cap = 0;
            return cuda_err("cudaMalloc(step buffers)", e);
        }
        *cap = c;
        return "";
    }

    void free_slots() {
        for (auto& sl : slots) {
            cudaFree(sl.d_tasks);
            cudaFree(sl.d_circs);
            cudaFree(sl.d_ctr);
            if (sl.h_tasks) cudaFreeHost(sl.h_tasks);
            if (sl.h_err) cudaFreeHost(sl.h_err);
            if (sl.ev) cudaEventDestroy(sl.ev);
            sl = Slot();
        }
        if (cstream) cudaStreamDestroy(cstream);
        cstream = nullptr;
    }

    bool has_work() const {
        for (const Req* r : live)
            if (r->next_level < r->levels) return true;
        return false;
    }

    // Builds the next step from the live requests' unscheduled levels and
    // queues it on the stream in slot `si`. Sets *launched when a step was
    // queued.
    std::string launch_step(int si, bool* launched) {
        *launched = false;
        Slot& S = slots[si];
        // Order: requests admitted more than a second ago first (no
        // starvation), then by remaining work (short jobs first).
        const double tnow = now();
        std::vector<std::pair<std::pair<int, int64_t>, Req*>> order;
        for (Req* r : live) {
            if (r->next_level >= r->levels) continue;
            int64_t rem = 0;
            for (int a = r->next_level; a < r->levels; a++) rem += level_cost(r, a);
            order.push_back({{tnow - r->t_admit > 1.0 ? 0 : 1, rem}, r});
        }
        std::stable_sort(order.begin(), order.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        std::vector<std::pair<Req*, int>> sched;  // request, levels this step
        int64_t used = 0;
        for (auto& it : order) {
            if ((int)sched.size() >= kMaxStepCircuits) break;
            Req* r = it.second;
            int L = 0;
            double chain = 0.0;
            while (r->next_level + L < r->levels) {
                const int64_t c = level_cost(r, r->next_level + L);
                const double lat = level_latency_us(r, r->next_level + L);
                if (L > 0 && opt.step_latency_us > 0 && chain + lat > opt.step_latency_us) break;
                if (used + c > opt.step_tiles && (L > 0 || used > 0)) break;
                used += c;
                chain += lat;
                L++;
            }
            if (L > 0) sched.push_back({r, L});
        }
        if (sched.empty()) return "";
        // Task list: requests grouped by tiles per pass (small groups first),
        // level-major inside a group.
        std::stable_sort(sched.begin(), sched.end(),
                         [](const auto& a, const auto& b) { return a.first->ncos < b.first->ncos; });
        std::vector<BatchCirc> circs;
        std::vector<BatchTask> tasks;
        std::vector<int> cnt(sched.size(), 0);
        for (size_t i = 0; i < sched.size(); i++) circs.push_back(sched[i].first->circ);
        size_t g0 = 0;
        const int chunk = std::max(1, opt.chunk), zch = std::max(1, opt.zchunks), sch = std::max(1, opt.schunks);
        while (g0 < sched.size()) {
            size_t g1 = g0;
            int maxL = 0;
            while (g1 < sched.size() && sched[g1].first->ncos == sched[g0].first->ncos) {
                maxL = std::max(maxL, sched[g1].second);
                g1++;
            }
            for (int l = 0; l < maxL; l++)
                for (size_t i = g0; i < g1; i++) {
                    Req* r = sched[i].first;
                    if (l >= sched[i].second) continue;
                    const int a = r->next_level + l;
                    const int before = cnt[i];
                    auto add = [&](int kind, uint32_t c0, uint32_t c1) {
                        BatchTask t{};
                        t.kind = kind;
                        t.circ = (int32_t)i;
                        t.c0 = c0;
                        t.c1 = c1;
                        t.need = before;
                        if (kind == BT_PASS) {
                            t.prog = (int32_t)(r->prog0 + a);
                            t.first = a == 0;
                        }
                        tasks.push_back(t);
                        cnt[i]++;
                    };
                    if (a < r->npass) {
                        // Small states: one coset per task, so a level spreads over several CTAs.
                        const uint32_t ch = std::max<uint32_t>(1, std::min<uint32_t>(chunk, r->ncos / 64));
                        for (uint32_t c0 = 0; c0 < r->ncos; c0 += ch) add(BT_PASS, c0, std::min(r->ncos, c0 + ch));
                    } else if (a == r->npass) {
                        for (uint32_t c0 = 0; c0 < r->nch; c0 += zch) add(BT_ZRED, c0, std::min(r->nch, c0 + zch));
                    } else if (a == r->npass + 1) {
                        add(BT_PREFIX, 0, 1);
                    } else {
                        for (uint32_t c0 = 0; c0 < r->nch; c0 += sch) add(BT_SAMPLE, c0, std::min(r->nch, c0 + sch));
                    }
                }
            g0 = g1;
        }
        if (tasks.size() > (size_t)INT32_MAX) return "step has too many tasks";
        std::string e = ensure((void**)&S.d_tasks, &S.tasks_cap, tasks.size() * sizeof(BatchTask));
        if (e.empty()) e = ensure((void**)&S.d_circs, &S.circs_cap, circs.size() * sizeof(BatchCirc));
        if (!e.empty()) return e;
        if (tasks.size() > S.h_tasks_cap) {
            // The slot's previous copy finished with its step.
            if (S.h_tasks) cudaFreeHost(S.h_tasks);
            S.h_tasks_cap = std::max(tasks.size(), 2 * S.h_tasks_cap);
            cudaError_t ce = cudaHostAlloc((void**)&S.h_tasks, S.h_tasks_cap * sizeof(BatchTask), cudaHostAllocDefault);
            if (ce != cudaSuccess) {
                S.h_tasks = nullptr;
                S.h_tasks_cap = 0;
                return cuda_err("cudaHostAlloc(tasks)", ce);
            }
        }
        std::memcpy(S.h_tasks, tasks.data(), tasks.size() * sizeof(BatchTask));
        cudaMemcpyAsync(S.d_tasks, S.h_tasks, tasks.size() * sizeof(BatchTask), cudaMemcpyHostToDevice, stream);
        cudaMemcpyAsync(S.d_circs, circs.data(), circs.size() * sizeof(BatchCirc), cudaMemcpyHostToDevice, stream);
        cudaMemsetAsync(S.d_ctr, 0, sizeof(int) * (2 + circs.size()), stream);
        const int g = (int)std::min<size_t>((size_t)grid, tasks.size());
        const double tb = now();
        us_build += (int64_t)((tb - tnow) * 1e6);
        cudaError_t le = launch_batch(d_state, precision, S.d_tasks, (int)tasks.size(), S.d_circs,
                                      reinterpret_cast<const BatchProg*>(d_aux), d_aux,
                                      reinterpret_cast<const DevOp*>(d_aux), d_aux, S.d_ctr, S.d_ctr + 2,
                                      reinterpret_cast<double*>(d_aux), S.d_ctr + 1, g, stream,
                                      reinterpret_cast<double*>(d_aux), reinterpret_cast<const double*>(d_aux),
                                      reinterpret_cast<uint64_t*>(d_aux), 5000000000ull,
                                      precision == 1 && opt.tune.blocks ? 1 : 0);
        if (le != cudaSuccess) return cuda_err("launch_batch", le);
        cudaEventRecord(S.ev, stream);
        S.t_launch = tb;
        S.finishing.clear();
        for (auto& x : sched) {
            x.first->next_level += x.second;
            if (x.first->next_level >= x.first->levels) S.finishing.push_back(x.first);
        }
        inflight.push_back(si);
        *launched = true;
        return "";
    }

    // Waits for the oldest queued step; returns the requests it finished.
    std::string complete_oldest(std::vector<Req*>& finished) {
        const int si = inflight.front();
        inflight.pop_front();
        Slot& S = slots[si];
        cudaError_t ce = cudaEventSynchronize(S.ev);
        us_kernel += (int64_t)((now() - std::max(S.t_launch, last_done)) * 1e6);
        last_done = now();
        if (ce != cudaSuccess) return cuda_err("cudaEventSynchronize(step)", ce);
        cudaStreamWaitEvent(cstream, S.ev, 0);
        cudaMemcpyAsync(S.h_err, S.d_ctr + 1, sizeof(int), cudaMemcpyDeviceToHost, cstream);
        ce = cudaStreamSynchronize(cstream);
        if (ce != cudaSuccess) return cuda_err("cudaStreamSynchronize(results)", ce);
        if (*S.h_err) return "serving step: a dependency wait timed out";
        n_steps++;
        finished = S.finishing;
        S.finishing.clear();
        return "";
    }
    double last_done = 0;

    std::vector<uint64_t> h_out;  // staging for results (pinned)
    uint64_t* h_pinned = nullptr;
    size_t h_pinned_cap = 0;

    // Copies the finished requests' <Z> and samples with one asynchronous
    // copy each and one synchronisation, then publishes the results.
    void collect(const std::vector<Req*>& fin) {
        size_t words = 0;
        for (Req* r : fin) words += (size_t)r->pack.n_out + r->shots;
        if (words > h_pinned_cap) {
            if (h_pinned) cudaFreeHost(h_pinned);
            h_pinned_cap = std::max(words, 2 * h_pinned_cap);
            if (cudaHostAlloc((void**)&h_pinned, h_pinned_cap * 8, cudaHostAllocDefault) != cudaSuccess) {
                h_pinned = nullptr;
                h_pinned_cap = 0;
            }
        }
        uint64_t* host = h_pinned;
        if (!host) {
            h_out.resize(words);
            host = h_out.data();
        }
        size_t o = 0;
        for (Req* r : fin) {
            const size_t w = (size_t)r->pack.n_out + r->shots;
            cudaMemcpyAsync(host + o, d_aux + 8 * r->zoff, 8 * w, cudaMemcpyDeviceToHost, cstream);
            o += w;
        }
        cudaStreamSynchronize(cstream);
        o = 0;
        for (Req* r : fin) {
            ServeResult res;
            res.n = r->pack.n_out;
            res.z.resize(res.n);
            std::memcpy(res.z.data(), host + o, 8 * res.n);
            const uint64_t* phys = host + o + res.n;
            o += (size_t)res.n + r->shots;
            res.samples.assign(phys, phys + r->shots);  // physical indices; wait() converts them
            res.zbit = r->pack.zbit;
            res.t_submit = r->t_submit;
            res.t_admit = r->t_admit;
            res.t_done = now();
            release(r);
            std::lock_guard<std::mutex> lk(m);
            results[r->id] = std::move(res);
            n_completed++;
        }
    }

    void engine_loop() {
        cudaSetDevice(device);
        for (;;) {
            // Admission, in submission order.
            std::vector<Req*> to_admit, failed;
            {
                std::unique_lock<std::mutex> lk(m);
                if (live.empty() && inflight.empty())
                    cv_engine.wait_for(lk, std::chrono::milliseconds(2), [&] {
                        if (stop) return true;
                        auto it = waiting.find(next_admit);
                        return it != waiting.end() && it->second->planned;
                    });
                if (stop) return;
            }
            for (;;) {
                Req* r = nullptr;
                {
                    std::lock_guard<std::mutex> lk(m);
                    auto it = waiting.find(next_admit);
                    if (it == waiting.end() || !it->second->planned) break;
                    r = it->second;
                }
                if (!r->pack.err.empty()) {
                    std::lock_guard<std::mutex> lk(m);
                    failures[r->id] = r->pack.err;
                    waiting.erase(r->id);
                    next_admit++;
                    n_failed++;
                    delete r;
                    cv_done.notify_all();
                    continue;
                }
                const uint64_t sbytes = (1ull << r->pack.n_sim) * amp_bytes();
                if (sbytes > opt.budget_bytes) {
                    std::lock_guard<std::mutex> lk(m);
                    failures[r->id] = "state exceeds the admission budget";
                    waiting.erase(r->id);
                    next_admit++;
                    n_failed++;
                    delete r;
                    cv_done.notify_all();
                    continue;
                }
                const double ta = now();
                const bool admitted = resident + sbytes <= opt.budget_bytes && admit(r);
                us_admit += (int64_t)((now() - ta) * 1e6);
                if (!admitted) {
                    if (!live.empty()) break;  // wait for memory to free up
                    std::lock_guard<std::mutex> lk(m);
                    failures[r->id] = "request does not fit the device arenas";
                    waiting.erase(r->id);
                    next_admit++;
                    n_failed++;
                    delete r;
                    cv_done.notify_all();
                    continue;
                }
                r->t_admit = now();
                std::lock_guard<std::mutex> lk(m);
                waiting.erase(r->id);
                next_admit++;
                live.push_back(r);
            }
            // Keep up to two steps queued: the next one is built while the
            // current one runs.
            std::string e;
            while (e.empty() && inflight.size() < 2 && has_work()) {
                bool launched = false;
                e = launch_step(slot_next, &launched);
                if (!launched) break;
                slot_next ^= 1;
            }
            std::vector<Req*> finished;
            if (e.empty()) {
                if (inflight.empty()) continue;  // nothing to run: back to waiting for arrivals
                e = complete_oldest(finished);
            }
            if (!e.empty()) {
                // Fail every live request; the engine keeps serving new ones.
                cudaStreamSynchronize(stream);
                inflight.clear();
                for (Slot& S : slots) S.finishing.clear();
                std::lock_guard<std::mutex> lk(m);
                for (Req* r : live) {
                    failures[r->id] = e;
                    n_failed++;
                    states.release(r->state_off);
                    aux.release(r->aux_off);
                    resident -= (1ull << r->pack.n_sim) * amp_bytes();
                    delete r;
                }
                live.clear();
                cv_done.notify_all();
                continue;
            }
            const double tc = now();
            if (!finished.empty()) collect(finished);
            for (Req* r : finished) {
                {
                    std::lock_guard<std::mutex> lk(m);
                    live.erase(std::find(live.begin(), live.end(), r));
                }
                delete r;
            }
            us_collect += (int64_t)((now() - tc) * 1e6);
            if (!finished.empty()) cv_done.notify_all();
        }
    }
};

std::string Server::create(int precision, int device, const ServeOptions& opt, Server** out) {
    if (precision != 0 && precision != 1) return "unknown precision";
    auto* S = new ServerImpl();
    S->device = device;
    S->precision = precision;
    S->opt = opt;
    S->t0 = std::chrono::steady_clock::now();
    auto fail = [&](const std::string& e) {
        cudaFree(S->d_state);
        cudaFree(S->d_aux);
        S->free_slots();
        if (S->stream) cudaStreamDestroy(S->stream);
        delete S;
        return e;
    };
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return fail(cuda_err("cudaSetDevice", ce));
    ce = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamCreate", ce));
    const uint64_t minb = (1ull << KATE_TILE_BITS) * S->amp_bytes();
    const uint64_t budget = opt.budget_bytes / minb * minb;
    if (budget < minb) return fail("admission budget below one 12-qubit state");
    release_cached(device);  // the budget is one allocation: no simulator state held back for reuse
    ce = cudaMalloc(&S->d_state, budget);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(state arena)", ce));
    ce = cudaMalloc((void**)&S->d_aux, opt.aux_bytes);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(aux arena)", ce));
    ce = cudaStreamCreateWithFlags(&S->cstream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamCreate", ce));
    for (auto& sl : S->slots) {
        ce = cudaMalloc((void**)&sl.d_ctr, sizeof(int) * (2 + ServerImpl::kMaxStepCircuits));
        if (ce == cudaSuccess) ce = cudaHostAlloc((void**)&sl.h_err, sizeof(int), cudaHostAllocDefault);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
        if (ce != cudaSuccess) return fail(cuda_err("step slot allocation", ce));
        cudaMemset(sl.d_ctr, 0, sizeof(int) * 2);
    }
    S->states.init(budget, minb, 22);
    S->aux.init(opt.aux_bytes);
    S->grid = batch_grid(device, precision, precision == 1 && opt.tune.blocks);
    const int np = opt.planners > 0 ? opt.planners
                                    : (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (int i = 0; i < np; i++) S->planners.emplace_back([S] { S->plan_loop(); });
    S->engine = std::thread([S] { S->engine_loop(); });
    auto* s = new Server();
    s->d_ = S;
    *out = s;
    return "";
}

Server::~Server() {
    if (!d_) return;
    {
        std::lock_guard<std::mutex> lk(d_->m);
        d_->stop = true;
    }
    d_->cv_plan.notify_all();
    d_->cv_engine.notify_all();
    d_->cv_done.notify_all();
    for (auto& t : d_->planners) t.join();
    if (d_->engine.joinable()) d_->engine.join();
    cudaSetDevice(d_->device);
    cudaStreamSynchronize(d_->stream);
    for (Req* r : d_->live) delete r;
    for (auto& kv : d_->waiting) delete kv.second;
    cudaFree(d_->d_state);
    cudaFree(d_->d_aux);
    d_->free_slots();
    if (d_->h_pinned) cudaFreeHost(d_->h_pinned);
    cudaStreamDestroy(d_->stream);
    delete d_;
}

std::string Server::submit(const Program& p, int shots, uint64_t seed, int64_t* id) {
    if (shots < 0 || shots > (1 << 24)) return "shots out of range";
    if (p.nqbits < KATE_TILE_BITS || p.nqbits > KATE_BATCH_MAX_QUBITS) return "served circuits have 12 to 28 qubits";
    auto* r = new Req();
    r->prog = p;
    r->shots = shots;
    r->seed = seed;
    {
        std::lock_guard<std::mutex> lk(d_->m);
        if (d_->live.size() + d_->waiting.size() >= 65536) {
            delete r;
            return "too many requests in flight";
        }
        r->id = d_->next_id++;
        r->t_submit = d_->now();
        d_->waiting[r->id] = r;
        d_->planq.push_back(r);
        d_->n_submitted++;
        *id = r->id;
    }
    d_->cv_plan.notify_one();
    return "";
}

std::string Server::wait(int64_t id, double timeout_s, ServeResult* out) {
    std::unique_lock<std::mutex> lk(d_->m);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    for (;;) {
        auto it = d_->results.find(id);
        if (it != d_->results.end()) {
            *out = std::move(it->second);
            d_->results.erase(it);
            lk.unlock();
            // Physical amplitude index -> program-label order.
            for (auto& v : out->samples) {
                uint64_t w = 0;
                for (int x = 0; x < out->n; x++) w |= ((v >> out->zbit[x]) & 1ull) << x;
                v = w;
            }
            return "";
        }
        auto f = d_->failures.find(id);
        if (f != d_->failures.end()) {
            std::string e = f->second;
            d_->failures.erase(f);
            return e;
        }
        if (id < 0 || id >= d_->next_id) return "unknown request id";
        if (d_->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            if (d_->results.count(id) || d_->failures.count(id)) continue;
            return "timeout";
        }
    }
}

void Server::stats(int64_t* out) const {
    std::lock_guard<std::mutex> lk(d_->m);
    out[0] = d_->n_submitted;
    out[1] = d_->n_completed;
    out[2] = (int64_t)d_->live.size();
    out[3] = (int64_t)d_->waiting.size();
    out[4] = d_->n_steps;
    out[5] = (int64_t)d_->resident.load();
    out[6] = (int64_t)d_->peak_resident.load();
    out[7] = d_->n_failed;
    out[8] = d_->us_admit.load();
    out[9] = d_->us_build.load();
    out[10] = d_->us_kernel.load();
    out[11] = d_->us_collect.load();
}

double Server::now() const { return d_->now(); }

}  // namespace kate
