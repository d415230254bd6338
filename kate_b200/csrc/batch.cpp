// Batched execution. See batch.hpp and k_batch.cu.
#include "batch.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <chrono>
#include <memory>
#include <thread>

#include "devcache.hpp"
#include "launch.hpp"
#include "plan.hpp"

namespace kate {

namespace {

std::string cuda_err(const char* what, cudaError_t e) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}
#define KCHECK(call)                                       \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_err(#call, e_); \
    } while (0)

const BatchTune kDefaultTune{};

uint64_t put_bytes(std::vector<uint8_t>& blob, const void* p, size_t bytes) {
    const size_t off = (blob.size() + 15) & ~size_t(15);
    blob.resize(off + bytes);
    if (bytes) std::memcpy(blob.data() + off, p, bytes);
    return off;
}

}  // namespace

std::string pack_circuit(const Program& in, const BatchTune& tune, bool resident, CircPack& out, bool c64) {
    Program p = in;
    const int n = p.nqbits;
    if (n < 1 || n > KATE_BATCH_MAX_QUBITS) return "batch circuits have 1 to 28 qubits";
    if (resident && n < KATE_TILE_BITS) return "resident circuits have at least 12 qubits";
    out.n_out = n;
    out.small = !resident && n <= KATE_BATCH_SMALL_MAX;
    std::string e;
    if (p.instructions.empty() && p.groups.empty() && tune.fusion >= 2) {
        e = pass_schedule(p);
        if (e.empty()) e = pass_fuse(p, tune.fusion, 1e-6);
        if (!e.empty()) return e;
    }
    if (n < KATE_TILE_BITS) {
        // Idle qubits n..11 fill the tile; they stay |0> and have no output.
        p.nqbits = KATE_TILE_BITS;
        if (!p.instructions.empty())
            for (int q = n; q < KATE_TILE_BITS; q++) {
                p.initial_permutation.push_back(q);
                p.final_inverse_permutation.push_back(q);
            }
    }
    if (p.instructions.empty()) {
        e = pass_compile_default(p, 0, p.nqbits);
        if (!e.empty()) return e;
    }
    out.n_sim = p.nqbits;
    PlanOptions o;
    o.max_tile = KATE_TILE_BITS;
    o.group_qubits = tune.group >= 6 && tune.group <= KATE_TILE_BITS ? tune.group : KATE_TILE_BITS;
    o.coalesce = tune.coalesce >= 1 && tune.coalesce <= 6 ? tune.coalesce : 4;
    o.remap = !out.small;  // a resident tile is never written back, so it keeps its layout
    o.fuse_1q = true;
    o.staged = true;
    o.c64 = false;
    o.max_gates_per_pass = std::max(1, tune.max_gates);
    // Tensor-core block passes for a complex64 state kept in HBM; a plan
    // with any pass the blocks cannot take keeps register-staged programs.
    Plan plan;
    out.blocks = false;
    if (c64 && tune.blocks && !out.small && out.n_sim >= KATE_TILE_BITS) {
        PlanOptions ob = o;
        ob.c64 = true;
        ob.staged = false;
        e = build_plan(p, ob, &plan);
        bool all = e.empty() && !plan.passes.empty();
        for (const PlannedPass& pp : plan.passes) all = all && pp.bprog != nullptr;
        out.blocks = all;
    }
    if (!out.blocks) {
        plan = Plan();
        e = build_plan(p, o, &plan);
        if (!e.empty()) return e;
    }
    for (int x = 0; x < n; x++) out.zbit.push_back((uint8_t)plan.final_phys[plan.label_to_logical[x]]);
    out.pool = plan.pool;
    out.sops = plan.smem_ops;
    auto header = [&](const PlannedPass* pp, BatchProg& bp) {
        if (pp) {
            DevPass dp = to_devpass(out.n_sim, *pp, 0);
            bp.m = dp.m;
            bp.ncb = dp.ncb;
            std::memcpy(bp.tphys, dp.tphys, 16);
            std::memcpy(bp.outsrc, dp.outsrc, 16);
            std::memcpy(bp.cphys, dp.cphys, 48);
        } else {  // identity pass on the natural layout
            bp.m = KATE_TILE_BITS;
            bp.ncb = out.n_sim - KATE_TILE_BITS;
            for (int t = 0; t < KATE_TILE_BITS; t++) bp.tphys[t] = bp.outsrc[t] = (uint8_t)t;
            for (int b = 0; b < bp.ncb; b++) bp.cphys[b] = (uint8_t)(KATE_TILE_BITS + b);
        }
    };
    for (const PlannedPass& pp : plan.passes) {
        BatchProg bp{};
        header(&pp, bp);
        if (bp.m != KATE_TILE_BITS) return "internal: batch pass tile is not 12 qubits";
        if (!out.small && bp.tphys[0] != 0) return "internal: batch pass tile does not hold physical bit 0";
        if (out.blocks) {
            BlockProg b = *pp.bprog;
            const uint64_t at = put_bytes(out.blob, &b, sizeof(BlockProg));
            for (int k = 0; k < b.nblocks; k++) {
                const uint64_t img = put_bytes(out.blob, plan.bimg.data() + pp.bprog->bimg[k], KATE_BLOCK_IMG_BYTES);
                b.bimg[k] = img - at;
            }
            std::memcpy(out.blob.data() + at, &b, sizeof(BlockProg));
            bp.flags = BPROG_BLOCK;
            bp.nstages = 0;
            bp.ops_off = at;
        } else if (pp.prog) {
            const PassProg& P = *pp.prog;
            bp.nops = P.nops;
            bp.nmats = P.nmats;
            bp.nstages = P.nstages;
            bp.sop0 = P.sop0;
            for (int k = 0; k < P.nops; k++)
                if (P.ops[k].kind == SOP_SMEM) bp.flags |= BPROG_SMEM;
            bp.ops_off = put_bytes(out.blob, P.ops, sizeof(SOp) * P.nops);
            bp.mats_off = put_bytes(out.blob, P.mats, sizeof(double) * 2 * P.nmats);
            bp.stab_off = put_bytes(out.blob, P.stab, sizeof(uint16_t) * 44 * P.nstages);
        } else {
            bp.nops = (int)pp.ops.size();
            bp.nstages = -1;
            bp.ops_off = put_bytes(out.blob, pp.ops.data(), sizeof(DevOp) * pp.ops.size());
            out.generic.push_back({bp.ops_off, bp.nops});
        }
        out.progs.push_back(bp);
    }
    if (out.progs.empty() && !out.small) {
        BatchProg bp{};
        header(nullptr, bp);
        out.progs.push_back(bp);
    }
    // Register-staged programs carry their own matrices; only shared-memory
    // ops and generic passes read the pool, so without them it is not sent.
    if (out.sops.empty() && out.generic.empty()) std::vector<Cx>().swap(out.pool);
    return "";
}

namespace {

// Runs f(i) for i in [0, count) on up to 32 host threads (one below 8 items).
template <typename F>
void for_each_item(size_t count, F f) {
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < count;) f(i);
    };
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 32u));
    if (count < 8) nt = 1;
    std::vector<std::thread> th;
    for (unsigned k = 1; k < nt; k++) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
}

// Plans every circuit on host threads.
std::vector<CircPack> pack_all(const std::vector<const Program*>& circuits, const BatchOptions& opt, bool c64) {
    std::vector<CircPack> packs(circuits.size());
    for_each_item(circuits.size(), [&](size_t i) {
        const BatchTune& tu = opt.for_n(circuits[i]->nqbits);
        try {
            packs[i].err = pack_circuit(*circuits[i], tu, false, packs[i], c64);
        } catch (const std::exception& ex) {
            packs[i].err = ex.what();
        }
    });
    return packs;
}

}  // namespace

const BatchTune& BatchOptions::for_n(int n) const {
    if (n >= 0 && (size_t)n < tune.size() && tune[n].fusion >= 1 && tune[n].max_gates >= 1) return tune[n];
    return kDefaultTune;
}

namespace {
// Times one candidate tuning for qubit count n on `sample`; ms < 0 when the
// candidate does not plan.
std::string time_candidate(const std::vector<const Program*>& sample, int precision, int device,
                           const BatchOptions& base, int n, const BatchTune& t, float* ms) {
    BatchOptions o = base;
    o.tune[n] = t;
    Batch* b = nullptr;
    *ms = -1.f;
    if (!Batch::create(sample, precision, device, o, &b).empty()) return "";
    std::string e = b->time_runs(1, ms);
    if (e.empty()) e = b->time_runs(3, ms);
    delete b;
    return e;
}
}  // namespace

struct BatchImpl {
    int device = 0;
    int precision = 1;
    int ncirc = 0;
    int64_t nout = 0;
    uint64_t arena_amps = 0;
    int grid = 0;
    std::vector<BatchTask> tasks;
    std::vector<BatchCirc> circs;
    std::vector<int> cprogs, cres;  // per circuit: programs, resident qubits
    std::vector<BatchProg> progs;
    std::unique_ptr<uint8_t[]> blob;  // concatenated program blobs (host copy, freed after upload)
    uint64_t blob_bytes = 0;
    std::vector<DevOp> sops;
    std::vector<Cx> pool;
    void* d_arena = nullptr;
    BatchTask* d_tasks = nullptr;
    BatchCirc* d_circs = nullptr;
    BatchProg* d_progs = nullptr;
    void* d_blob = nullptr;
    DevOp* d_sops = nullptr;
    void* d_pool = nullptr;
    int* d_head = nullptr;
    int* d_done = nullptr;
    double* d_zout = nullptr;
    int* d_err = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double create_ms[4] = {0, 0, 0, 0};  // planning, assembly, device buffers + uploads, graph
    uint64_t upload_bytes = 0;           // host-to-device bytes copied by create()
    uint64_t wait_ns = 5000000000ull;    // a dependency wait in the kernel gives up after this long
    bool tensor_blocks = false;          // some circuit runs tensor-core block passes
    int64_t block_programs = 0;          // pass programs run as tensor-core block passes

    size_t amp_bytes() const { return precision == 0 ? 16 : 8; }

    void release() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cached_free(d_arena, device);
        cudaFree(d_tasks);
        cudaFree(d_circs);
        cudaFree(d_progs);
        cudaFree(d_blob);
        cudaFree(d_sops);
        cudaFree(d_pool);
        cudaFree(d_head);
        cudaFree(d_done);
        cudaFree(d_zout);
        cudaFree(d_err);
        if (stream) cudaStreamDestroy(stream);
        exec = nullptr;
        graph = nullptr;
        stream = nullptr;
    }

    template <typename T>
    std::string upload(T** dptr, const std::vector<T>& v, const char* what) {
        const size_t bytes = std::max<size_t>(16, v.size() * sizeof(T));
        cudaError_t e = cudaMalloc((void**)dptr, bytes);
        if (e != cudaSuccess) return cuda_err(what, e);
        if (!v.empty()) {
            e = cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return cuda_err(what, e);
        }
        return "";
    }
};

std::string Batch::create(const std::vector<const Program*>& circuits, int precision, int device,
                          const BatchOptions& opt, Batch** out) {
    if (precision != 0 && precision != 1) return "unknown precision";
    if (circuits.empty()) return "empty batch";
    for (const Program* p : circuits)
        if (!p) return "null circuit";
    const int chunk = std::max(1, opt.chunk), zchunks = std::max(1, opt.zchunks);
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
    clk::time_point t0 = clk::now();
    std::vector<CircPack> packs = pack_all(circuits, opt, precision == 1);
    const double plan_ms = ms_since(t0);
    t0 = clk::now();
    for (size_t i = 0; i < packs.size(); i++)
        if (!packs[i].err.empty()) return "circuit " + std::to_string(i) + ": " + packs[i].err;

    auto* S = new BatchImpl();
    auto fail = [&](const std::string& e) {
        S->release();
        delete S;
        return e;
    };
    S->device = device;
    S->precision = precision;
    S->ncirc = (int)circuits.size();
    S->create_ms[0] = plan_ms;

    // Concatenate the packs: offsets first, then every pack copied in
    // parallel into buffers allocated once (uninitialised, so each page is
    // first touched by the thread that fills it). Large states are laid out
    // in the arena in circuit order.
    const size_t np = packs.size();
    std::vector<uint64_t> boff(np), poff(np), soff(np);
    std::vector<int> prog0(np);
    {
        uint64_t bsz = 0, psz = 0, ssz = 0, gsz = 0;
        S->circs.resize(np);
        S->cprogs.resize(np);
        S->cres.resize(np);
        for (size_t i = 0; i < np; i++) {
            const CircPack& P = packs[i];
            bsz = (bsz + 15) & ~uint64_t(15);
            boff[i] = bsz;
            bsz += P.blob.size();
            poff[i] = psz;
            psz += P.pool.size();
            soff[i] = ssz;
            ssz += P.sops.size();
            prog0[i] = (int)gsz;
            gsz += P.progs.size();
            BatchCirc bc{};
            bc.n = P.n_out;
            bc.zoff = S->nout;
            bc.poff = -1;
            S->nout += P.n_out;
            for (int x = 0; x < P.n_out; x++) bc.zbit[x] = P.zbit[x];
            if (!P.small) {
                bc.off = S->arena_amps;
                S->arena_amps += 1ull << P.n_sim;
            }
            S->circs[i] = bc;
            S->tensor_blocks = S->tensor_blocks || P.blocks;
            if (P.blocks) S->block_programs += (int64_t)P.progs.size();
            S->cprogs[i] = (int)P.progs.size();
            S->cres[i] = P.small ? 0 : P.n_sim;
        }
        if (ssz > (uint64_t)INT32_MAX || gsz > (uint64_t)INT32_MAX) return fail("too many programs or shared-memory ops");
        S->blob_bytes = std::max<uint64_t>(16, bsz);
        S->blob.reset(new uint8_t[S->blob_bytes]);
        S->pool.resize(psz);
        S->sops.resize(ssz);
        S->progs.resize(gsz);
    }
    for_each_item(np, [&](size_t i) {
        CircPack& P = packs[i];
        uint8_t* bl = S->blob.get() + boff[i];
        const uint64_t end = i + 1 < np ? boff[i + 1] : S->blob_bytes;
        if (!P.blob.empty()) std::memcpy(bl, P.blob.data(), P.blob.size());
        std::memset(bl + P.blob.size(), 0, end - boff[i] - P.blob.size());  // alignment padding
        const int64_t pbase = (int64_t)poff[i];
        for (auto& g : P.generic) {
            DevOp* ops = reinterpret_cast<DevOp*>(bl + g.first);
            for (int k = 0; k < g.second; k++) ops[k].mat += pbase;
        }
        DevOp* so = S->sops.data() + soff[i];
        for (size_t k = 0; k < P.sops.size(); k++) {
            so[k] = P.sops[k];
            so[k].mat += pbase;
        }
        std::copy(P.pool.begin(), P.pool.end(), S->pool.begin() + (ptrdiff_t)poff[i]);
        BatchProg* pr = S->progs.data() + prog0[i];
        for (size_t k = 0; k < P.progs.size(); k++) {
            BatchProg bp = P.progs[k];
            bp.ops_off += boff[i];
            bp.mats_off += boff[i];
            bp.stab_off += boff[i];
            bp.sop0 += (int)soff[i];
            pr[k] = bp;
        }
        std::vector<uint8_t>().swap(P.blob);
        std::vector<Cx>().swap(P.pool);
        std::vector<DevOp>().swap(P.sops);
    });

    // Task queue. Large circuits, window by window, level by level; small
    // circuits spread evenly between them (they depend on nothing, so they
    // fill the waits at level boundaries): small circuit s goes right after
    // the first L*s/Sn large tasks, L large tasks in all.
    std::vector<int> large, small;
    for (size_t i = 0; i < np; i++) (packs[i].small ? small : large).push_back((int)i);
    auto pass_tasks = [&](const CircPack& P) -> uint64_t {
        const uint32_t ncos = 1u << (P.n_sim - KATE_TILE_BITS);
        const uint32_t cch = std::max<uint32_t>(1, std::min<uint32_t>(chunk, ncos / 16));
        return (ncos + cch - 1) / cch;
    };
    auto zred_tasks = [&](const CircPack& P) -> uint64_t {
        const uint64_t nch = std::max<uint64_t>(1, (1ull << P.n_sim) >> 16);
        return (nch + zchunks - 1) / zchunks;
    };
    uint64_t L = 0;
    for (int ci : large) L += pass_tasks(packs[ci]) * packs[ci].progs.size() + zred_tasks(packs[ci]);
    const uint64_t Sn = small.size();
    if (L + Sn > (uint64_t)INT32_MAX) return fail("too many tasks");
    S->tasks.reserve(L + Sn);
    uint64_t li = 0, si = 0;
    auto push_small = [&]() {
        BatchTask st{};
        st.kind = BT_SMALL;
        st.circ = small[si];
        st.prog = prog0[small[si]];
        st.nprog = (int)packs[small[si]].progs.size();
        S->tasks.push_back(st);
        si++;
    };
    auto push_large = [&](const BatchTask& t) {
        while (si < Sn && L * si / Sn <= li) push_small();
        S->tasks.push_back(t);
        li++;
    };
    {
        size_t w0 = 0;
        std::vector<int> need(large.size(), 0);
        while (w0 < large.size()) {
            size_t w1 = w0;
            uint64_t bytes = 0;
            do {
                bytes += (1ull << packs[large[w1]].n_sim) * S->amp_bytes();
                w1++;
            } while (w1 < large.size() && (opt.window_bytes == 0 ||
                                           bytes + (1ull << packs[large[w1]].n_sim) * S->amp_bytes() <= opt.window_bytes));
            size_t maxlev = 0;
            for (size_t k = w0; k < w1; k++) maxlev = std::max(maxlev, packs[large[k]].progs.size() + 1);
            for (size_t lev = 0; lev < maxlev; lev++)
                for (size_t k = w0; k < w1; k++) {
                    const int ci = large[k];
                    const CircPack& P = packs[ci];
                    const size_t nprog = P.progs.size();
                    if (lev > nprog) continue;
                    const int before = need[k];
                    if (lev < nprog) {
                        const uint32_t ncos = 1u << (P.n_sim - KATE_TILE_BITS);
                        // Small states: fewer cosets per task, so a level spreads over several CTAs.
                        const uint32_t cch = std::max<uint32_t>(1, std::min<uint32_t>(chunk, ncos / 16));
                        for (uint32_t c0 = 0; c0 < ncos; c0 += cch) {
                            BatchTask t{};
                            t.kind = BT_PASS;
                            t.circ = ci;
                            t.prog = prog0[ci] + (int)lev;
                            t.c0 = c0;
                            t.c1 = std::min<uint32_t>(ncos, c0 + cch);
                            t.need = before;
                            t.first = lev == 0;
                            push_large(t);
                            need[k]++;
                        }
                    } else {
                        const uint32_t nch = (uint32_t)std::max<uint64_t>(1, (1ull << P.n_sim) >> 16);
                        for (uint32_t c0 = 0; c0 < nch; c0 += zchunks) {
                            BatchTask t{};
                            t.kind = BT_ZRED;
                            t.circ = ci;
                            t.c0 = c0;
                            t.c1 = std::min<uint32_t>(nch, c0 + zchunks);
                            t.need = before;
                            push_large(t);
                            need[k]++;
                        }
                    }
                }
            w0 = w1;
        }
        while (si < Sn) push_small();  // only when there are no large circuits
    }
    if (li != L) return fail("internal: task count mismatch");
    // Test hook: one task waits for a count its circuit never reaches, so the
    // kernel's bounded wait runs out (the failure is made on the host).
    if (opt.fault_task >= 0 && (size_t)opt.fault_task < S->tasks.size()) S->tasks[opt.fault_task].need = INT32_MAX;
    S->wait_ns = 1000000ull * (uint64_t)std::max(1, opt.wait_ms);
    S->create_ms[1] = ms_since(t0);
    t0 = clk::now();

    // Device side.
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return fail(cuda_err("cudaSetDevice", ce));
    ce = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamCreate", ce));
    std::string e;
    if ((e = S->upload(&S->d_tasks, S->tasks, "cudaMalloc(tasks)")) != "") return fail(e);
    if ((e = S->upload(&S->d_circs, S->circs, "cudaMalloc(circuits)")) != "") return fail(e);
    if ((e = S->upload(&S->d_progs, S->progs, "cudaMalloc(programs)")) != "") return fail(e);
    if ((e = S->upload(&S->d_sops, S->sops, "cudaMalloc(smem ops)")) != "") return fail(e);
    {
        ce = cudaMalloc(&S->d_blob, S->blob_bytes);
        if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(program blob)", ce));
        ce = cudaMemcpy(S->d_blob, S->blob.get(), S->blob_bytes, cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return fail(cuda_err("cudaMemcpy(program blob)", ce));
        Cx* p = nullptr;
        if ((e = S->upload(&p, S->pool, "cudaMalloc(matrix pool)")) != "") return fail(e);
        S->d_pool = p;
    }
    ce = cached_malloc(&S->d_arena, std::max<uint64_t>(16, S->arena_amps * S->amp_bytes()), device);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(state arena)", ce));
    ce = cudaMalloc((void**)&S->d_head, sizeof(int));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(queue head)", ce));
    ce = cudaMalloc((void**)&S->d_done, sizeof(int) * S->ncirc);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(counters)", ce));
    ce = cudaMalloc((void**)&S->d_zout, sizeof(double) * std::max<int64_t>(1, S->nout));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(outputs)", ce));
    ce = cudaMalloc((void**)&S->d_err, sizeof(int));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(error flag)", ce));
    ce = cudaMemset(S->d_err, 0, sizeof(int));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMemset(error flag)", ce));
    S->upload_bytes = S->tasks.size() * sizeof(BatchTask) + S->circs.size() * sizeof(BatchCirc) +
                      S->progs.size() * sizeof(BatchProg) + S->sops.size() * sizeof(DevOp) + S->blob_bytes +
                      S->pool.size() * sizeof(Cx);
    S->grid = batch_grid(device, precision, S->tensor_blocks);
    const int grid = (int)std::min<size_t>((size_t)S->grid, S->tasks.size());
    S->create_ms[2] = ms_since(t0);
    t0 = clk::now();

    // One graph: reset queue, counters and outputs, then the kernel.
    ce = cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamBeginCapture", ce));
    cudaMemsetAsync(S->d_head, 0, sizeof(int), S->stream);
    cudaMemsetAsync(S->d_done, 0, sizeof(int) * S->ncirc, S->stream);
    cudaMemsetAsync(S->d_zout, 0, sizeof(double) * std::max<int64_t>(1, S->nout), S->stream);
    cudaError_t le = launch_batch(S->d_arena, precision, S->d_tasks, (int)S->tasks.size(), S->d_circs, S->d_progs,
                                  S->d_blob, S->d_sops, S->d_pool, S->d_head, S->d_done, S->d_zout, S->d_err, grid,
                                  S->stream, nullptr, nullptr, nullptr, S->wait_ns, S->tensor_blocks ? 1 : 0);
    ce = cudaStreamEndCapture(S->stream, &S->graph);
    if (le != cudaSuccess) return fail(cuda_err("launch_batch", le));
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamEndCapture", ce));
    ce = cudaGraphInstantiate(&S->exec, S->graph, 0);
    if (ce != cudaSuccess) return fail(cuda_err("cudaGraphInstantiate", ce));
    S->create_ms[3] = ms_since(t0);
    // Host copies are no longer needed.
    S->blob.reset();
    std::vector<Cx>().swap(S->pool);
    std::vector<DevOp>().swap(S->sops);
    auto* b = new Batch();
    b->d_ = S;
    *out = b;
    return "";
}

Batch::~Batch() {
    if (!d_) return;
    d_->release();
    delete d_;
}

std::string Batch::run_async(void* stream) {
    KCHECK(cudaSetDevice(d_->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : d_->stream;
    KCHECK(cudaGraphLaunch(d_->exec, st));
    if (st != d_->stream) {
        cudaEvent_t ev;
        KCHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        KCHECK(cudaEventRecord(ev, st));
        KCHECK(cudaStreamWaitEvent(d_->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    return "";
}

std::string Batch::synchronize() {
    KCHECK(cudaSetDevice(d_->device));
    KCHECK(cudaStreamSynchronize(d_->stream));
    int err = 0;
    KCHECK(cudaMemcpy(&err, d_->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        cudaMemset(d_->d_err, 0, sizeof(int));
        return "batch kernel: a dependency wait timed out; outputs are incomplete";
    }
    return "";
}

std::string Batch::expect_z(double* out) {
    std::string e = synchronize();
    if (!e.empty()) return e;
    KCHECK(cudaMemcpy(out, d_->d_zout, sizeof(double) * d_->nout, cudaMemcpyDeviceToHost));
    return "";
}

std::string Batch::time_runs(int runs, float* ms_avg) {
    KCHECK(cudaSetDevice(d_->device));
    cudaEvent_t a, b;
    KCHECK(cudaEventCreate(&a));
    KCHECK(cudaEventCreate(&b));
    KCHECK(cudaEventRecord(a, d_->stream));
    for (int r = 0; r < runs; r++) KCHECK(cudaGraphLaunch(d_->exec, d_->stream));
    KCHECK(cudaEventRecord(b, d_->stream));
    std::string e = synchronize();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (!e.empty()) return e;
    *ms_avg = ms / std::max(1, runs);
    return "";
}

int64_t Batch::num_outputs() const { return d_->nout; }
int64_t Batch::num_tasks() const { return (int64_t)d_->tasks.size(); }
uint64_t Batch::arena_bytes() const { return d_->arena_amps * d_->amp_bytes(); }
int Batch::grid() const { return d_->grid; }
void Batch::create_times(double* ms4) const {
    for (int k = 0; k < 4; k++) ms4[k] = d_->create_ms[k];
}
uint64_t Batch::upload_bytes() const { return d_->upload_bytes; }
int64_t Batch::num_programs() const { return (int64_t)d_->progs.size(); }
int64_t Batch::num_block_programs() const { return d_->block_programs; }
void Batch::circuit_info(int i, int* programs, int* resident_qubits) const {
    *programs = d_->cprogs[i];
    *resident_qubits = d_->cres[i];
}

std::string Batch::get_state(int i, double* out) {
    BatchImpl& B = *d_;
    if (i < 0 || i >= B.ncirc) return "circuit index out of range";
    if (B.cres[i] == 0)
        return "circuit " + std::to_string(i) + " ran in one CTA's shared memory and has no resident state";
    const BatchCirc& C = B.circs[i];
    const int n = C.n;                   // the circuit's qubits (outputs)
    const uint64_t dim = 1ull << n;
    const uint64_t dim_sim = 1ull << B.cres[i];  // amplitudes kept (padding qubits stay 0)
    std::vector<uint8_t> h(dim_sim * B.amp_bytes());
    cudaError_t ce = cudaSetDevice(B.device);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(B.stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(h.data(), (const uint8_t*)B.d_arena + C.off * B.amp_bytes(), h.size(), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return std::string("batch state: ") + cudaGetErrorString(ce);
    // Label index x has qubit q at physical bit zbit[q].
    for (uint64_t x = 0; x < dim; x++) {
        uint64_t p = 0;
        for (int q = 0; q < n; q++) p |= ((x >> q) & 1ull) << C.zbit[q];
        if (p >= dim_sim) return "internal: output bit outside the resident state";
        if (B.precision == 1) {
            const float* f = reinterpret_cast<const float*>(h.data()) + 2 * p;
            out[2 * x] = f[0];
            out[2 * x + 1] = f[1];
        } else {
            const double* d = reinterpret_cast<const double*>(h.data()) + 2 * p;
            out[2 * x] = d[0];
            out[2 * x + 1] = d[1];
        }
    }
    return "";
}

std::string batch_autotune(const std::vector<const Program*>& circuits, int precision, int device,
                           BatchOptions* opt) {
    if (opt->tune.size() < KATE_BATCH_MAX_QUBITS + 1) opt->tune.resize(KATE_BATCH_MAX_QUBITS + 1, BatchTune{0, 0, 0, 0, 0});
    std::map<int, std::vector<const Program*>> byn;
    for (const Program* p : circuits)
        if (p) byn[p->nqbits].push_back(p);
    static const int kFusion[] = {1, 2, 3};
    static const int kGates[] = {64, 96, 128};
    static const int kGroup[] = {11, 10};
    static const int kCoalesce[] = {3, 5};
    for (auto& kv : byn) {
        const int n = kv.first;
        const int nsim = std::max(n, KATE_TILE_BITS);
        // A sample of about 2^27 amplitudes of state (at most 512 circuits).
        size_t cnt = (size_t)std::max<uint64_t>(1, (1ull << 27) >> nsim);
        cnt = std::min<size_t>({cnt, kv.second.size(), 512});
        std::vector<const Program*> sample(kv.second.begin(), kv.second.begin() + cnt);
        float best = 0.f;
        BatchTune bt = kDefaultTune;
        bool found = false;
        auto consider = [&](const BatchTune& t) -> std::string {
            float ms = 0.f;
            std::string e = time_candidate(sample, precision, device, *opt, n, t, &ms);
            if (!e.empty()) return e;
            if (ms >= 0.f && (!found || ms < best)) {
                best = ms;
                bt = t;
                found = true;
            }
            return "";
        };
        // Coordinate search: fusion width x gates per pass at the default
        // grouping and coalescing, then the grouping size m, then the
        // coalesce width c (which only matters for states kept in HBM).
        for (int f : kFusion)
            for (int g : kGates) {
                std::string e = consider(BatchTune{f, g, KATE_TILE_BITS, 4});
                if (!e.empty()) return e;
            }
        if (!found) return "autotune: no candidate plan for " + std::to_string(n) + "-qubit circuits";
        for (int m : kGroup) {
            BatchTune t = bt;
            t.group = m;
            std::string e = consider(t);
            if (!e.empty()) return e;
        }
        if (n > KATE_BATCH_SMALL_MAX)
            for (int c : kCoalesce) {
                BatchTune t = bt;
                t.coalesce = c;
                std::string e = consider(t);
                if (!e.empty()) return e;
            }
        // Complex64 states kept in HBM: tensor-core blocks (the planner
        // forms them, so no prior gateFusion) with the chosen grouping and
        // coalescing, and with the defaults.
        if (precision == 1 && n > KATE_BATCH_SMALL_MAX) {
            const BatchTune cand[2] = {BatchTune{1, bt.max_gates, bt.group, bt.coalesce, 1},
                                       BatchTune{1, kDefaultTune.max_gates, KATE_TILE_BITS, 4, 1}};
            for (const BatchTune& t : cand) {
                std::string e = consider(t);
                if (!e.empty()) return e;
            }
        }
        opt->tune[n] = bt;
    }
    return "";
}

}  // namespace kate
