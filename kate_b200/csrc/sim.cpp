// Device simulator. See sim.hpp.
#include "sim.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>

#include "devcache.hpp"
#include "jit.hpp"
#include "launch.hpp"

namespace kate {

namespace {
constexpr double kPi = 3.1415926535897932384626433;
constexpr double kSqrt2 = 1.4142135623730951;

std::string cuda_err(const char* what, cudaError_t e) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}
#define KCHECK(call)                                              \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_err(#call, e_);        \
    } while (0)
}  // namespace

struct SimImpl {
    int device = 0;
    int n = 0;
    int precision = 0;
    Program prog;
    Plan plan;
    PlanOptions opt;
    void* d_state = nullptr;
    DevOp* d_ops = nullptr;
    DevOp* d_sops = nullptr;   // shared-memory ops of register-staged programs
    void* d_pool = nullptr;
    void* d_part = nullptr;
    void* d_bimg = nullptr;   // complex64 block operand images
    int* d_err = nullptr;     // set by kernels whose bounded waits gave up
    void* d_norm = nullptr;   // complex64: renormalisation scratch and result
    bool renormed = false;    // a complex64 run has been renormalised
    size_t part_bytes = 0;
    std::vector<DevPass> hpasses;
    cudaStream_t stream = nullptr;
    std::vector<int> phys;  // current layout: logical -> physical
    bool has_state = false;
    int grid = 0;
    int tile_grid = 0;
    int nbuf = 1;  // tile kernel buffering (1: two CTAs per SM, 2: one CTA, prefetching)
    int ws_grid = 0;
    std::vector<char> ws_ok;  // pass i runs on the warp-specialised complex128 tile kernel
    std::vector<void*> jit_fn;  // pass i runs on its pass-specialised kernel (complex128)
    void* jit_fn0 = nullptr;    // pass 0 generating its input |0...0> (no initialisation pass)
    bool zero_start = false;    // the run being enqueued starts with jit_fn0
    void* jit_fnP = nullptr;    // pass 0 computing a product-state input (no initialisation pass)
    bool prod_start = false;    // the run being enqueued starts with jit_fnP and prod_tab
    ProdTab prod_tab{};
    int jit_grid_n = 0;

    // Launches pass i of the plan on stream st.
    cudaError_t launch_pass(size_t i, cudaStream_t st) {
        const PlannedPass& p = plan.passes[i];
        if (p.bprog) return launch_block_c64(d_state, *p.bprog, d_bimg, d_err, block_grid, st);
        if (i == 0 && zero_start && jit_fn0) return jit_launch(jit_fn0, d_state, *p.prog, jit_grid_n, st);
        if (i == 0 && prod_start && jit_fnP) return jit_launch_prod(jit_fnP, d_state, *p.prog, prod_tab, jit_grid_n, st);
        if (p.prog && i < jit_fn.size() && jit_fn[i]) return jit_launch(jit_fn[i], d_state, *p.prog, jit_grid_n, st);
        if (p.prog && i < ws_ok.size() && ws_ok[i]) return launch_tile_ws(d_state, *p.prog, d_err, ws_grid, st);
        if (p.prog) return launch_tile(d_state, precision, *p.prog, d_sops, d_pool, tile_grid, nbuf, st);
        return launch_pass_generic(d_state, precision, hpasses[i], d_ops, d_pool, grid, st);
    }
    int block_grid = 0;

    uint64_t dim() const { return 1ull << n; }
    size_t amp_bytes() const { return precision == 0 ? 16 : 8; }

    // Target layout for readback: label x at physical bit x.
    std::vector<int> label_layout() const {
        std::vector<int> t(n);
        for (int x = 0; x < n; x++) t[plan.label_to_logical[x]] = x;
        return t;
    }
    // Physical bit of program label x.
    int phys_of_label(int x) const { return phys[plan.label_to_logical[x]]; }

    std::string run_relayout(const std::vector<int>& target) {
        if (phys == target) return "";
        std::vector<PlannedPass> pp = plan_relayout(n, phys, target, opt);
        for (auto& p : pp) {
            DevPass d = to_devpass(n, p, 0);
            int grid_r = generic_pass_grid(n, d.m, device);
            KCHECK(launch_pass_generic(d_state, precision, d, d_ops, d_pool, grid_r, stream));
        }
        phys = target;
        return "";
    }

    // Sums over amplitudes (kind 0) or probabilities (kind 1) for every
    // physical bit; s0/s1 are 2 doubles per bit for kind 0, 1 for kind 1.
    std::string bit_sums(int kind, std::vector<double>& s0, std::vector<double>& s1, double* total) {
        BitSumShape sh = bitsum_shape(n);
        const int w = kind == 0 ? 2 : 1;
        std::vector<double> h((size_t)sh.grid * sh.nout * w);
        KCHECK(launch_bitsums(d_state, precision, n, kind, d_part, stream));
        KCHECK(cudaMemcpyAsync(h.data(), d_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
        KCHECK(cudaStreamSynchronize(stream));
        s0.assign((size_t)n * w, 0.0);
        s1.assign((size_t)n * w, 0.0);
        std::vector<double> tot(w, 0.0);
        for (int c = 0; c < sh.grid; c++) {
            const double* pc = h.data() + (size_t)c * sh.nout * w;
            for (int k = 0; k < w; k++) tot[k] += pc[k];
            for (int b = 0; b < n; b++) {
                int slot;
                if (b < 12) slot = b;
                else if (b < 12 + sh.g) {
                    bool one = (c >> (b - 12)) & 1;
                    for (int k = 0; k < w; k++) (one ? s1 : s0)[(size_t)b * w + k] += pc[k];
                    continue;
                } else slot = 12 + (b - 12 - sh.g);
                for (int k = 0; k < w; k++) {
                    s0[(size_t)b * w + k] += pc[(size_t)(1 + 2 * slot) * w + k];
                    s1[(size_t)b * w + k] += pc[(size_t)(2 + 2 * slot) * w + k];
                }
            }
        }
        if (total) for (int k = 0; k < w; k++) total[k] = tot[k];
        return "";
    }
};

std::string Simulator::create(const Program& prog_in, int precision, int device, Simulator** out) {
    if (precision != 0 && precision != 1) return "unknown precision";
    if (prog_in.nqbits < 1 || prog_in.nqbits > 34) return "the device simulator supports 1 to 34 qubits";
    auto* impl = new SimImpl();
    auto fail = [&](const std::string& e) {
        auto* s = new Simulator();
        s->d_ = impl;
        delete s;
        return e;
    };
    impl->device = device;
    impl->n = prog_in.nqbits;
    impl->precision = precision;
    impl->prog = prog_in;
    if (impl->prog.instructions.empty()) {
        std::string e = pass_compile_default(impl->prog, 0, impl->prog.nqbits);
        if (!e.empty()) return fail(e);
    }
    impl->opt.c64 = precision == 1;
    {
        // Dense two-qubit gates as register ops for complex128, where the
        // pass-specialised kernels run them straight-line.
        const char* jv = std::getenv("KATE_JIT");
        impl->opt.dense2_reg = precision == 0 && !(jv && std::atoi(jv) == 0);
    }
    // Complex128 passes of 27 qubits and more choose the qubits they move
    // into the low bits by trying every subset, and the gate cap per pass
    // among a few (about 15 ms of planning for a 30-qubit, 1780-gate
    // circuit; below 27 qubits a pass takes under 0.7 ms and the search
    // would cost more host time than it saves). KATE_REMAP_SEARCH=0 or 1
    // forces it off or on.
    {
        const char* rs = std::getenv("KATE_REMAP_SEARCH");
        const bool on = rs ? std::atoi(rs) != 0 : prog_in.nqbits >= 27;
        impl->opt.remap_search = precision == 0 && on;
        impl->opt.cap_search = impl->opt.remap_search;
    }
    // Contiguous low physical bits every tile holds (runs of 2^c amplitudes per access).
    if (const char* e = std::getenv("KATE_COALESCE")) {
        const int v = std::atoi(e);
        if (v >= 1 && v <= 8) impl->opt.coalesce = v;
    }
    // Gates a pass may take at most (the planner packs greedily up to it).
    if (const char* e = std::getenv("KATE_MAX_GATES")) {
        const int v = std::atoi(e);
        if (v >= 1 && v <= 160) impl->opt.max_gates_per_pass = v, impl->opt.cap_search = false;
    }
    std::string e = build_plan(impl->prog, impl->opt, &impl->plan);
    if (!e.empty()) return fail(e);

    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return fail(cuda_err("cudaSetDevice", ce));
    ce = cudaStreamCreateWithFlags(&impl->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(cuda_err("cudaStreamCreate", ce));
    // Upload ops and the matrix pool.
    std::vector<DevOp> ops;
    for (auto& p : impl->plan.passes) {
        impl->hpasses.push_back(to_devpass(impl->n, p, (int)ops.size()));
        ops.insert(ops.end(), p.ops.begin(), p.ops.end());
    }
    size_t ops_bytes = std::max<size_t>(1, ops.size()) * sizeof(DevOp);
    size_t pool_bytes = std::max<size_t>(1, impl->plan.pool.size()) * sizeof(Cx);
    ce = cudaMalloc(&impl->d_ops, ops_bytes);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(ops)", ce));
    ce = cudaMalloc(&impl->d_pool, pool_bytes);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(pool)", ce));
    ce = cudaMalloc(&impl->d_sops, std::max<size_t>(1, impl->plan.smem_ops.size()) * sizeof(DevOp));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(smem ops)", ce));
    if (!impl->plan.smem_ops.empty())
        cudaMemcpy(impl->d_sops, impl->plan.smem_ops.data(), impl->plan.smem_ops.size() * sizeof(DevOp),
                   cudaMemcpyHostToDevice);
    if (!ops.empty()) cudaMemcpy(impl->d_ops, ops.data(), ops.size() * sizeof(DevOp), cudaMemcpyHostToDevice);
    if (!impl->plan.pool.empty())
        cudaMemcpy(impl->d_pool, impl->plan.pool.data(), impl->plan.pool.size() * sizeof(Cx), cudaMemcpyHostToDevice);
    ce = cudaMalloc(&impl->d_bimg, std::max<size_t>(16, impl->plan.bimg.size()));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(block images)", ce));
    if (!impl->plan.bimg.empty())
        cudaMemcpy(impl->d_bimg, impl->plan.bimg.data(), impl->plan.bimg.size(), cudaMemcpyHostToDevice);
    if (precision == 1) {
        ce = cudaMalloc(&impl->d_norm, renorm_scratch_bytes());
        if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(renormalisation)", ce));
        cudaMemset(impl->d_norm, 0, renorm_scratch_bytes());
    }
    ce = cudaMalloc(&impl->d_err, sizeof(int));
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(error flag)", ce));
    cudaMemset(impl->d_err, 0, sizeof(int));
    BitSumShape sh = bitsum_shape(impl->n);
    impl->part_bytes = (size_t)sh.grid * sh.nout * 2 * sizeof(double);
    ce = cudaMalloc(&impl->d_part, impl->part_bytes);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(partials)", ce));
    ce = cached_malloc(&impl->d_state, impl->dim() * impl->amp_bytes(), device);
    if (ce != cudaSuccess) return fail(cuda_err("cudaMalloc(state)", ce));
    impl->grid = generic_pass_grid(impl->n, std::min(impl->opt.max_tile, impl->n), device);
    if (const char* e = std::getenv("KATE_TILE_NBUF")) {
        const int v = std::atoi(e);
        impl->nbuf = v == 2 ? 2 : v == 3 ? 3 : 1;
    }
    if (impl->n >= KATE_TILE_BITS) {
        impl->tile_grid = tile_pass_grid(impl->n, device, impl->nbuf, precision);
        const char* jv = std::getenv("KATE_JIT");
        if (precision == 0 && !(jv && std::atoi(jv) == 0)) {
            // Pass-specialised kernels for every register-staged pass whose
            // program the generator takes; the others keep the interpreter.
            // Two CTAs per SM (at most 128 registers). KATE_JIT_OCC=3 asks
            // for three (at most 80 registers; a kernel that would spill
            // stays at two): measured slower on the layered workload (54.6
            // against 56.8 layers/s), kept as a tuning option.
            const char* oe = std::getenv("KATE_JIT_OCC");
            const int occ_force = oe ? std::atoi(oe) : 0;
            const int occ_first = occ_force == 3 ? 3 : 2;
            // Kernels per (pass, form): form 0 loads its input, form 1 (pass
            // 0) generates |0...0>, form 2 (pass 0) computes a product state.
            // Kernels compiled before for the same pass shape are found by
            // key; only the others get their source generated.
            std::vector<size_t> idx;
            std::vector<int> forms;
            std::vector<std::string> todo;
            std::vector<void*> fns;
            std::vector<std::string> keys;
            std::vector<size_t> miss;
            auto want = [&](size_t i, int form, int occ) {
                std::string key = jit_pass_key(*impl->plan.passes[i].prog, form, occ);
                void* f = jit_find(device, key);
                idx.push_back(i);
                forms.push_back(form);
                if (!f) {
                    miss.push_back(fns.size());
                    todo.push_back(jit_pass_source(*impl->plan.passes[i].prog, nullptr, form, occ));
                }
                fns.push_back(f);
                keys.push_back(std::move(key));
            };
            for (size_t i = 0; i < impl->plan.passes.size(); i++) {
                const PlannedPass& p = impl->plan.passes[i];
                if (!p.prog || p.bprog) continue;
                want(i, 0, occ_first);
            }
            if (!idx.empty() && idx[0] == 0) {
                want(0, 1, occ_first);
                want(0, 2, occ_first);
            }
            auto compile_missing = [&]() -> std::string {
                // Sources the generator declined stay null: those passes keep the interpreter.
                std::vector<std::string> srcs;
                std::vector<size_t> at;
                for (size_t m = 0; m < miss.size(); m++)
                    if (!todo[m].empty()) {
                        srcs.push_back(std::move(todo[m]));
                        at.push_back(miss[m]);
                    }
                std::vector<void*> got;
                std::string je = jit_compile(device, srcs, &got);
                if (!je.empty()) return je;
                for (size_t m = 0; m < at.size(); m++) {
                    fns[at[m]] = got[m];
                    jit_remember(device, keys[at[m]], got[m]);
                }
                miss.clear();
                todo.clear();
                return "";
            };
            std::string je = compile_missing();
            if (!je.empty()) return fail("pass kernel compilation: " + je);
            if (occ_first == 3) {
                // A kernel that spills at three CTAs per SM goes back to two.
                for (size_t k = 0; k < fns.size(); k++)
                    if (fns[k] && jit_local_bytes(fns[k]) != 0) {
                        std::string key = jit_pass_key(*impl->plan.passes[idx[k]].prog, forms[k], 2);
                        void* f = jit_find(device, key);
                        if (!f) {
                            miss.push_back(k);
                            todo.push_back(jit_pass_source(*impl->plan.passes[idx[k]].prog, nullptr, forms[k], 2));
                        }
                        fns[k] = f;
                        keys[k] = std::move(key);
                    }
                je = compile_missing();
                if (!je.empty()) return fail("pass kernel compilation: " + je);
            }
            impl->jit_fn.assign(impl->plan.passes.size(), nullptr);
            for (size_t k = 0; k < idx.size(); k++) {
                if (!fns[k]) continue;
                if (forms[k] == 0) impl->jit_fn[idx[k]] = fns[k];
                else if (forms[k] == 1) impl->jit_fn0 = fns[k];
                else impl->jit_fnP = fns[k];
            }
            // The start forms only serve when pass 0 itself has a kernel.
            if (impl->jit_fn.empty() || !impl->jit_fn[0]) impl->jit_fn0 = impl->jit_fnP = nullptr;
            impl->jit_grid_n = jit_grid(impl->n - KATE_TILE_BITS, device);
        }
        const char* ws = std::getenv("KATE_TILE_WS");
        if (precision == 0 && ws && std::atoi(ws) == 1) {
            impl->ws_grid = tile_ws_grid(impl->n, device);
            impl->ws_ok.assign(impl->plan.passes.size(), 0);
            for (size_t i = 0; i < impl->plan.passes.size(); i++) {
                const PlannedPass& p = impl->plan.passes[i];
                impl->ws_ok[i] = p.prog && !p.bprog && tile_ws_applies(*p.prog);
            }
        }
        if (precision == 1) impl->block_grid = block_c64_grid(impl->n, device);
    }
    impl->phys.resize(impl->n);
    std::iota(impl->phys.begin(), impl->phys.end(), 0);
    auto* s = new Simulator();
    s->d_ = impl;
    *out = s;
    return "";
}

Simulator::~Simulator() {
    if (!d_) return;
    cudaSetDevice(d_->device);
    if (d_->stream) cudaStreamSynchronize(d_->stream);
    cached_free(d_->d_state, d_->device);
    cudaFree(d_->d_ops);
    cudaFree(d_->d_sops);
    cudaFree(d_->d_pool);
    cudaFree(d_->d_part);
    cudaFree(d_->d_bimg);
    cudaFree(d_->d_err);
    cudaFree(d_->d_norm);
    if (d_->stream) cudaStreamDestroy(d_->stream);
    delete d_;
}

int Simulator::nqbits() const { return d_->n; }
int Simulator::precision() const { return d_->precision; }
const Plan& Simulator::plan() const { return d_->plan; }

std::string Simulator::run_async(void* stream_in, const double* tp) {
    SimImpl& S = *d_;
    KCHECK(cudaSetDevice(S.device));
    cudaStream_t st = stream_in ? (cudaStream_t)stream_in : S.stream;
    std::string e = enqueue_init(st, tp);
    if (!e.empty()) return e;
    e = enqueue_passes(st);
    if (!e.empty()) return e;
    if (st != S.stream) {
        // Order later library work on the simulator's stream after the caller's.
        cudaEvent_t ev;
        KCHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        KCHECK(cudaEventRecord(ev, st));
        KCHECK(cudaStreamWaitEvent(S.stream, ev, 0));
        cudaEventDestroy(ev);
    }
    return "";
}

std::string Simulator::enqueue_init(void* stream, const double* tp) {
    SimImpl& S = *d_;
    cudaStream_t st = (cudaStream_t)stream;
    if (tp) {
        // execute(proba_state&): product state, qubit i placed at label
        // initial_permutation[i] (CPUcode/simulator.hpp:139-162).
        ProductInit P{};
        P.n = S.n;
        for (int i = 0; i < S.n; i++) {
            double c0 = std::cos(tp[2 * i] * kPi / 2), s0 = std::sin(tp[2 * i] * kPi / 2);
            double er = std::cos(tp[2 * i + 1]), ei = std::sin(tp[2 * i + 1]);
            int lab = S.plan.initial_permutation.empty() ? i : S.plan.initial_permutation[i];
            P.v[0][lab][0] = c0;
            P.v[0][lab][1] = 0.0;
            P.v[1][lab][0] = er * s0;
            P.v[1][lab][1] = ei * s0;
        }
        S.prod_start = false;
        if (S.jit_fnP && !S.hpasses.empty()) {
            // The first pass computes the product state itself (no
            // initialisation pass, and the state is not read).
            for (int b = 0; b < 2; b++)
                for (int p = 0; p < S.n; p++) S.prod_tab.v[b][p] = make_double2(P.v[b][p][0], P.v[b][p][1]);
            S.prod_start = true;
            S.zero_start = false;
            return "";
        }
        KCHECK(launch_init_product(S.d_state, S.n, P, S.precision, st));
    } else if (S.jit_fn0) {
        // The first pass writes the whole state from |0...0> itself.
        S.zero_start = true;
        S.prod_start = false;
        return "";
    } else {
        KCHECK(launch_set_basis0(S.d_state, S.dim(), S.precision, st));
    }
    S.zero_start = false;
    S.prod_start = false;
    return "";
}

std::string Simulator::enqueue_passes(void* stream) {
    SimImpl& S = *d_;
    cudaStream_t st = (cudaStream_t)stream;
    const bool zs = S.zero_start, ps = S.prod_start;
    S.zero_start = S.prod_start = false;
    if (zs && S.hpasses.empty()) KCHECK(launch_set_basis0(S.d_state, S.dim(), S.precision, st));
    for (size_t i = 0; i < S.hpasses.size(); i++) {
        S.zero_start = zs && i == 0;
        S.prod_start = ps && i == 0;
        const cudaError_t ce = S.launch_pass(i, st);
        S.zero_start = S.prod_start = false;
        KCHECK(ce);
    }
    if (S.precision == 1) {
        // Complex64: ||psi|| in FP64, then the state rescaled to norm 1.
        KCHECK(launch_renorm_c64(S.d_state, S.n, S.d_norm, st));
        S.renormed = true;
    }
    S.phys = S.plan.final_phys;
    S.has_state = true;
    return "";
}

namespace {
struct EventSet {
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    ~EventSet() {
        for (auto x : e)
            if (x) cudaEventDestroy(x);
    }
};
}  // namespace

std::string Simulator::execute_timed(const double* tp_in, double* tp_out, double* ms) {
    SimImpl& S = *d_;
    KCHECK(cudaSetDevice(S.device));
    EventSet ev;
    for (auto& x : ev.e) KCHECK(cudaEventCreate(&x));
    KCHECK(cudaEventRecord(ev.e[0], S.stream));
    std::string e = enqueue_init(S.stream, tp_in);
    if (!e.empty()) return e;
    KCHECK(cudaEventRecord(ev.e[1], S.stream));
    e = enqueue_passes(S.stream);
    if (!e.empty()) return e;
    KCHECK(cudaEventRecord(ev.e[2], S.stream));
    e = synchronize();
    if (!e.empty()) return e;
    float a = 0, b = 0;
    KCHECK(cudaEventElapsedTime(&a, ev.e[0], ev.e[1]));
    KCHECK(cudaEventElapsedTime(&b, ev.e[1], ev.e[2]));
    const auto t0 = std::chrono::steady_clock::now();
    if (tp_out) {
        e = proba_state(tp_out);
        if (!e.empty()) return e;
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (ms) {
        ms[0] = a;
        ms[1] = b;
        ms[2] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        ms[3] = (double)S.hpasses.size();
    }
    return "";
}

std::string Simulator::synchronize() {
    KCHECK(cudaSetDevice(d_->device));
    KCHECK(cudaStreamSynchronize(d_->stream));
    int flag = 0;
    KCHECK(cudaMemcpy(&flag, d_->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(d_->d_err, 0, sizeof(int));
        return "timed out: a bounded device wait gave up (tensor-core completion not observed)";
    }
    return "";
}

std::string Simulator::proba_state(double* out) {
    SimImpl& S = *d_;
    if (!S.has_state) return "no state: execute the simulator first";
    KCHECK(cudaSetDevice(S.device));
    std::vector<double> s0, s1;
    std::string e = S.bit_sums(0, s0, s1, nullptr);
    if (!e.empty()) return e;
    // HIPcode/simulator.hpp:519-535 with the reference's Complex division,
    // norm and angle (backendagnosticcode/basic_host_types.hpp:28-57).
    const int n = S.n;
    const double p = std::pow(kSqrt2, (double)n);
    auto cdiv = [](double ar, double ai, double br, double bi, double& rr, double& ri) {
        double d = br * br + bi * bi;
        rr = (ar * br + ai * bi) / d;
        ri = (br * ai - ar * bi) / d;
    };
    for (int x = 0; x < n; x++) {
        int b = S.phys_of_label(x);
        double v0r, v0i, v1r, v1i;
        cdiv(s0[2 * b], s0[2 * b + 1], p, 0.0, v0r, v0i);
        cdiv(s1[2 * b], s1[2 * b + 1], p, 0.0, v1r, v1i);
        double n0 = std::sqrt(v0r * v0r + v0i * v0i), n1 = std::sqrt(v1r * v1r + v1i * v1i);
        double teta, phi;
        if (n0 < 0.0000000000001) {
            teta = 1;
            phi = 0;
        } else if (n1 < 0.00000000000001) {
            teta = 0;
            phi = 0;
        } else {
            teta = std::atan(n1 / n0) / (kPi / 2);
            double qr, qi;
            cdiv(v1r, v1i, v0r, v0i, qr, qi);
            phi = std::atan(qi / qr);
        }
        int o = S.plan.final_inverse_permutation.empty() ? x : S.plan.final_inverse_permutation[x];
        out[2 * o] = teta;
        out[2 * o + 1] = phi;
    }
    return "";
}

std::string Simulator::expect_z(double* out) {
    SimImpl& S = *d_;
    if (!S.has_state) return "no state: execute the simulator first";
    KCHECK(cudaSetDevice(S.device));
    std::vector<double> s0, s1;
    std::string e = S.bit_sums(1, s0, s1, nullptr);
    if (!e.empty()) return e;
    for (int x = 0; x < S.n; x++) {
        int b = S.phys_of_label(x);
        out[x] = s0[b] - s1[b];
    }
    return "";
}

std::string Simulator::get_state(double* out) {
    SimImpl& S = *d_;
    if (!S.has_state) return "no state: execute the simulator first";
    KCHECK(cudaSetDevice(S.device));
    std::string e = S.run_relayout(S.label_layout());
    if (!e.empty()) return e;
    if (S.precision == 0) {
        KCHECK(cudaMemcpyAsync(out, S.d_state, S.dim() * 16, cudaMemcpyDeviceToHost, S.stream));
        KCHECK(cudaStreamSynchronize(S.stream));
        return "";
    }
    // complex64: copy as floats, widen in place from the end of the buffer.
    float* f = reinterpret_cast<float*>(out);
    KCHECK(cudaMemcpyAsync(f, S.d_state, S.dim() * 8, cudaMemcpyDeviceToHost, S.stream));
    KCHECK(cudaStreamSynchronize(S.stream));
    for (uint64_t i = 2 * S.dim(); i-- > 0;) out[i] = (double)f[i];
    return "";
}

std::string Simulator::set_state(const double* in) {
    SimImpl& S = *d_;
    KCHECK(cudaSetDevice(S.device));
    if (S.precision == 0) {
        KCHECK(cudaMemcpyAsync(S.d_state, in, S.dim() * 16, cudaMemcpyHostToDevice, S.stream));
        KCHECK(cudaStreamSynchronize(S.stream));
    } else {
        std::vector<float> f(2 * S.dim());
        for (size_t i = 0; i < f.size(); i++) f[i] = (float)in[i];
        KCHECK(cudaMemcpyAsync(S.d_state, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice, S.stream));
        KCHECK(cudaStreamSynchronize(S.stream));
    }
    S.phys = S.label_layout();
    S.has_state = true;
    return "";
}

std::string Simulator::probabilities(double* out) {
    SimImpl& S = *d_;
    if (!S.has_state) return "no state: execute the simulator first";
    if (S.n > 30) return "probabilities are limited to 30 qubits";
    KCHECK(cudaSetDevice(S.device));
    std::string e = S.run_relayout(S.label_layout());
    if (!e.empty()) return e;
    double* d = nullptr;
    KCHECK(cudaMallocAsync((void**)&d, S.dim() * sizeof(double), S.stream));
    cudaError_t ce = launch_probs(S.d_state, S.precision, S.dim(), d, S.stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(out, d, S.dim() * sizeof(double), cudaMemcpyDeviceToHost, S.stream);
    cudaFreeAsync(d, S.stream);
    if (ce != cudaSuccess) return cuda_err("probabilities", ce);
    KCHECK(cudaStreamSynchronize(S.stream));
    return "";
}

std::string Simulator::sample(int shots, uint64_t seed, uint64_t* out) {
    SimImpl& S = *d_;
    if (shots < 0) return "shots must be >= 0";
    if (!S.has_state) return "no state: execute the simulator first";
    if (shots == 0) return "";
    KCHECK(cudaSetDevice(S.device));
    // Uniforms u = (splitmix64 >> 11) * 2^-53 in draw order (the generator
    // the server's samples use), sorted for the device with their shot index.
    std::vector<std::pair<double, int>> us((size_t)shots);
    uint64_t sm = seed;
    for (int k = 0; k < shots; k++) {
        sm += 0x9E3779B97F4A7C15ull;
        uint64_t z = sm;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        us[(size_t)k] = {(double)(z >> 11) * (1.0 / 9007199254740992.0), k};
    }
    std::sort(us.begin(), us.end());
    std::vector<double> u((size_t)shots);
    for (int k = 0; k < shots; k++) u[(size_t)k] = us[(size_t)k].first;
    const size_t nscr = sample_scratch_doubles(S.n);
    char* buf = nullptr;
    const size_t bytes = (nscr + (size_t)shots) * sizeof(double) + (size_t)shots * sizeof(uint64_t);
    KCHECK(cudaMallocAsync((void**)&buf, bytes, S.stream));
    double* d_scr = (double*)buf;
    double* d_u = d_scr + nscr;
    uint64_t* d_out = (uint64_t*)(d_u + shots);
    std::vector<uint64_t> phys((size_t)shots);
    cudaError_t ce = cudaMemcpyAsync(d_u, u.data(), (size_t)shots * sizeof(double), cudaMemcpyHostToDevice, S.stream);
    if (ce == cudaSuccess) ce = launch_sample(S.d_state, S.precision, S.n, d_u, shots, d_scr, d_out, S.stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(phys.data(), d_out, (size_t)shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, S.stream);
    cudaFreeAsync(buf, S.stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(S.stream);
    if (ce != cudaSuccess) return cuda_err("sample", ce);
    // Physical index -> index in the reference's qubit labels.
    std::vector<int> pb(S.n);
    for (int x = 0; x < S.n; x++) pb[x] = S.phys_of_label(x);
    for (int k = 0; k < shots; k++) {
        const uint64_t v = phys[(size_t)k];
        uint64_t lab = 0;
        for (int x = 0; x < S.n; x++) lab |= ((v >> pb[x]) & 1ull) << x;
        out[us[(size_t)k].second] = lab;
    }
    return "";
}

std::string Simulator::profile_passes(float* ms, float* init_ms) {
    SimImpl& S = *d_;
    KCHECK(cudaSetDevice(S.device));
    std::vector<cudaEvent_t> ev(S.hpasses.size() + 2);
    for (auto& e : ev) KCHECK(cudaEventCreate(&e));
    KCHECK(cudaEventRecord(ev[0], S.stream));
    KCHECK(launch_set_basis0(S.d_state, S.dim(), S.precision, S.stream));
    KCHECK(cudaEventRecord(ev[1], S.stream));
    for (size_t i = 0; i < S.hpasses.size(); i++) {
        KCHECK(S.launch_pass(i, S.stream));
        KCHECK(cudaEventRecord(ev[i + 2], S.stream));
    }
    KCHECK(cudaEventSynchronize(ev.back()));
    if (init_ms) KCHECK(cudaEventElapsedTime(init_ms, ev[0], ev[1]));
    for (size_t i = 0; i < S.hpasses.size(); i++) KCHECK(cudaEventElapsedTime(&ms[i], ev[i + 1], ev[i + 2]));
    for (auto& e : ev) cudaEventDestroy(e);
    S.phys = S.plan.final_phys;
    S.has_state = true;
    return "";
}

int Simulator::launches_per_run() const {
    return (d_->jit_fn0 ? 0 : 1) + (int)d_->hpasses.size() + (d_->precision == 1 ? 2 : 0);
}

std::string Simulator::norm2_before_renorm(double* out) {
    SimImpl& S = *d_;
    if (S.precision != 1) return "only complex64 simulators are renormalised";
    if (!S.renormed) return "no run has been renormalised yet";
    KCHECK(cudaSetDevice(S.device));
    KCHECK(cudaStreamSynchronize(S.stream));
    KCHECK(cudaMemcpy(out, (const char*)S.d_norm + renorm_result_offset(), sizeof(double), cudaMemcpyDeviceToHost));
    return "";
}

int Simulator::pass_kernel(int i) const {
    const SimImpl& S = *d_;
    if (i < 0 || i >= (int)S.plan.passes.size()) return -1;
    const PlannedPass& p = S.plan.passes[i];
    if (p.bprog) return 3;
    if (p.prog && (size_t)i < S.jit_fn.size() && S.jit_fn[i]) return 2;
    if (p.prog) return 1;
    return 0;
}

bool Simulator::pass_work(int i, double out[3]) const {
    if (pass_kernel(i) != 2) return false;
    out[0] = 2.0 * 16.0;
    return jit_pass_work(*d_->plan.passes[i].prog, &out[1], &out[2]);
}

std::string Simulator::state_device(void** dptr, int* phys) {
    *dptr = d_->d_state;
    for (int x = 0; x < d_->n; x++) phys[x] = d_->phys_of_label(x);
    return "";
}

}  // namespace kate
