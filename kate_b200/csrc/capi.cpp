// C ABI (include/kate_b200.h) over the C++ circuit, passes and simulator.
#include "devcache.hpp"
#include "kate_b200.h"

#include <cuda_runtime.h>

#include <cstring>
#include <exception>
#include <string>

#include "batch.hpp"
#include "circuit.hpp"
#include "plan.hpp"
#include "serve.hpp"
#include "jit.hpp"
#include "launch.hpp"
#include "sim.hpp"

struct kate_circuit {
    kate::Program prog;
};
struct kate_sim {
    kate::Simulator* sim = nullptr;
};
struct kate_batch {
    kate::Batch* b = nullptr;
    int ncirc = 0;
};
struct kate_server {
    kate::Server* s = nullptr;
};
struct kate_plan {
    kate::Plan plan;
    std::vector<DevPass> passes;
    std::vector<DevOp> ops;
};

namespace {
thread_local std::string g_last_error;

kate_status fail(kate_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

kate_status from_msg(const std::string& msg, kate_status code = KATE_EINVAL) {
    if (msg.empty()) return KATE_OK;
    return fail(code, msg);
}

// Simulator messages from CUDA calls carry the call name; classify them.
// A bounded device wait that gave up says "timed out".
kate_status sim_status(const std::string& msg) {
    if (msg.empty()) return KATE_OK;
    if (msg.find("timed out") != std::string::npos) return fail(KATE_ETIMEDOUT, msg);
    if (msg.find("cudaMalloc") != std::string::npos || msg.find("MemoryAllocation") != std::string::npos)
        return fail(KATE_ENOMEM, msg);
    if (msg.find("no state") != std::string::npos) return fail(KATE_ESTATE, msg);
    if (msg.find("cuda") != std::string::npos || msg.find("launch") != std::string::npos)
        return fail(KATE_ECUDA, msg);
    return fail(KATE_EINVAL, msg);
}

// Errors of device work already queued: a bounded wait that gave up, else
// a CUDA failure.
kate_status device_status(const std::string& msg) {
    if (msg.empty()) return KATE_OK;
    if (msg.find("timed out") != std::string::npos) return fail(KATE_ETIMEDOUT, msg);
    return fail(KATE_ECUDA, msg);
}

template <typename F>
kate_status guarded(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return fail(KATE_ENOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(KATE_EINVAL, e.what());
    }
}

#define REQUIRE(cond, msg) \
    if (!(cond)) return fail(KATE_EINVAL, msg)
}  // namespace

namespace kate {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace kate

extern "C" {

const char* kate_last_error(void) { return g_last_error.c_str(); }
const char* kate_version(void) { return "kate_b200 0.1 (sm_100a)"; }

kate_status kate_device_count(int* out) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();  // no driver or no device: report zero devices
        n = 0;
    }
    if (out) *out = n;
    return KATE_OK;
}

kate_status kate_device_properties(int device, char* name, int name_cap, size_t* global_mem,
                                   size_t* shared_mem_per_block, int* sm_count) {
    int n = 0;
    kate_device_count(&n);
    REQUIRE(device >= 0 && device < n, "no such CUDA device");
    cudaDeviceProp p{};
    const cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) return fail(KATE_ECUDA, std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
    if (name && name_cap > 0) {
        std::strncpy(name, p.name, (size_t)name_cap - 1);
        name[name_cap - 1] = 0;
    }
    if (global_mem) *global_mem = p.totalGlobalMem;
    if (shared_mem_per_block) *shared_mem_per_block = p.sharedMemPerBlock;
    if (sm_count) *sm_count = p.multiProcessorCount;
    return KATE_OK;
}

kate_status kate_circuit_create(int nqbits, kate_circuit** out) {
    return guarded([&] {
        REQUIRE(out, "null output pointer");
        REQUIRE(nqbits >= 1 && nqbits <= KATE_MAX_QUBITS, "nqbits must be in [1, 40]");
        auto* c = new kate_circuit();
        c->prog.nqbits = nqbits;
        *out = c;
        return KATE_OK;
    });
}

kate_status kate_circuit_destroy(kate_circuit* c) {
    delete c;
    return KATE_OK;
}

kate_status kate_circuit_clone(const kate_circuit* c, kate_circuit** out) {
    return guarded([&] {
        REQUIRE(c && out, "null pointer");
        *out = new kate_circuit(*c);
        return KATE_OK;
    });
}

kate_status kate_circuit_nqbits(const kate_circuit* c, int* out) {
    REQUIRE(c && out, "null pointer");
    *out = c->prog.nqbits;
    return KATE_OK;
}

kate_status kate_circuit_append_gate(kate_circuit* c, int id, const int* qbits, int nq, int optarg) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        REQUIRE(nq >= 0 && nq <= 64 && (nq == 0 || qbits), "bad qubit list");
        if (id == kate::G_DENSE) return fail(KATE_EINVAL, "use kate_circuit_append_dense for dense gates");
        kate::Gate g;
        g.id = id;
        g.qbits.assign(qbits, qbits + nq);
        g.optarg = optarg;
        std::string e = kate::validate_gate(c->prog, g);
        if (!e.empty()) return fail(e.find("after gateGrouping") != std::string::npos ? KATE_ESTATE : KATE_EINVAL, e);
        c->prog.gates.push_back(std::move(g));
        return KATE_OK;
    });
}

kate_status kate_circuit_append_dense(kate_circuit* c, const double* mat, const int* qbits, int nq) {
    return guarded([&] {
        REQUIRE(c && mat && qbits, "null pointer");
        REQUIRE(nq >= 1 && nq <= 10, "dense gates take 1 to 10 qubits");
        kate::Gate g;
        g.id = kate::G_DENSE;
        g.qbits.assign(qbits, qbits + nq);
        size_t len = (size_t)1 << (2 * nq);
        g.dense.resize(len);
        for (size_t i = 0; i < len; i++) g.dense[i] = kate::Cx(mat[2 * i], mat[2 * i + 1]);
        std::string e = kate::validate_gate(c->prog, g);
        if (!e.empty()) return fail(e.find("after gateGrouping") != std::string::npos ? KATE_ESTATE : KATE_EINVAL, e);
        c->prog.gates.push_back(std::move(g));
        return KATE_OK;
    });
}

kate_status kate_circuit_append_many(kate_circuit* c, int count, const int* ids, const int* nqs, const int* qbits,
                                     const int* optargs, const double* dense) {
    return guarded([&] {
        REQUIRE(c && count >= 0, "null pointer");
        if (count == 0) return KATE_OK;
        REQUIRE(ids && nqs && qbits, "null pointer");
        kate::Program tmp;
        tmp.nqbits = c->prog.nqbits;
        std::vector<kate::Gate> add;
        add.reserve(count);
        size_t qo = 0, dofs = 0;
        for (int i = 0; i < count; i++) {
            const int nq = nqs[i];
            REQUIRE(nq >= 1 && nq <= 10, "gates take 1 to 10 qubits");
            kate::Gate g;
            g.id = ids[i];
            g.qbits.assign(qbits + qo, qbits + qo + nq);
            qo += nq;
            g.optarg = optargs ? optargs[i] : 0;
            if (g.id == kate::G_DENSE) {
                REQUIRE(dense, "dense gates need matrix entries");
                const size_t len = (size_t)1 << (2 * nq);
                g.dense.resize(len);
                for (size_t k = 0; k < len; k++) g.dense[k] = kate::Cx(dense[2 * (dofs + k)], dense[2 * (dofs + k) + 1]);
                dofs += len;
                g.optarg = 0;
            }
            std::string e = kate::validate_gate(c->prog, g);
            if (!e.empty())
                return fail(e.find("after gateGrouping") != std::string::npos ? KATE_ESTATE : KATE_EINVAL,
                            "gate " + std::to_string(i) + ": " + e);
            add.push_back(std::move(g));
        }
        for (auto& g : add) c->prog.gates.push_back(std::move(g));
        return KATE_OK;
    });
}

kate_status kate_circuit_num_gates(const kate_circuit* c, int* out) {
    REQUIRE(c && out, "null pointer");
    *out = (int)c->prog.gates.size();
    return KATE_OK;
}

kate_status kate_circuit_get_gate(const kate_circuit* c, int i, int* id, int* qbits, int* nq, int* optarg,
                                  double* dense) {
    REQUIRE(c && id && qbits && nq && optarg, "null pointer");
    REQUIRE(i >= 0 && i < (int)c->prog.gates.size(), "gate index out of range");
    const kate::Gate& g = c->prog.gates[i];
    *id = g.id;
    *nq = (int)g.qbits.size();
    for (size_t k = 0; k < g.qbits.size(); k++) qbits[k] = g.qbits[k];
    *optarg = g.optarg;
    if (dense && g.id == kate::G_DENSE)
        for (size_t k = 0; k < g.dense.size(); k++) {
            dense[2 * k] = g.dense[k].re;
            dense[2 * k + 1] = g.dense[k].im;
        }
    return KATE_OK;
}

kate_status kate_circuit_schedule(kate_circuit* c) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        return from_msg(kate::pass_schedule(c->prog));
    });
}

kate_status kate_circuit_fuse(kate_circuit* c, int k, double mtm) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        REQUIRE(k >= 1, "qbitsizelimit must be >= 1");
        kate::Program tmp = c->prog;
        std::string e = kate::pass_fuse(tmp, k, mtm);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        c->prog = std::move(tmp);
        return KATE_OK;
    });
}

kate_status kate_circuit_group(kate_circuit* c, int m) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        REQUIRE(m >= 1, "qbitgroupsize must be >= 1");
        return from_msg(kate::pass_group(c->prog, m));
    });
}

kate_status kate_circuit_allocate(kate_circuit* c, int g, int maxlocal) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        kate::Program tmp = c->prog;
        std::string e = kate::pass_allocate(tmp, g, maxlocal);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        c->prog = std::move(tmp);
        return KATE_OK;
    });
}

kate_status kate_circuit_compile_default(kate_circuit* c, int g, int maxlocal) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        kate::Program tmp = c->prog;
        std::string e = kate::pass_compile_default(tmp, g, maxlocal);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        c->prog = std::move(tmp);
        return KATE_OK;
    });
}

kate_status kate_circuit_compile_opt(kate_circuit* c, int k, double mtm, int groupsize, int g, int maxlocal) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        kate::Program tmp = c->prog;
        std::string e = kate::pass_schedule(tmp);
        if (e.empty()) e = kate::pass_fuse(tmp, k, mtm);
        if (e.empty()) e = kate::pass_group(tmp, groupsize);
        if (e.empty()) e = kate::pass_allocate(tmp, g, maxlocal);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        c->prog = std::move(tmp);
        return KATE_OK;
    });
}

kate_status kate_circuit_num_groups(const kate_circuit* c, int* out) {
    REQUIRE(c && out, "null pointer");
    *out = (int)c->prog.groups.size();
    return KATE_OK;
}

kate_status kate_circuit_get_group(const kate_circuit* c, int i, int* end, int* qbits, int* nq) {
    REQUIRE(c && end && qbits && nq, "null pointer");
    REQUIRE(i >= 0 && i < (int)c->prog.groups.size(), "group index out of range");
    auto& g = c->prog.groups[i];
    *end = g.first;
    *nq = (int)g.second.size();
    for (size_t k = 0; k < g.second.size(); k++) qbits[k] = g.second[k];
    return KATE_OK;
}

kate_status kate_circuit_num_instructions(const kate_circuit* c, int* out) {
    REQUIRE(c && out, "null pointer");
    *out = (int)c->prog.instructions.size();
    return KATE_OK;
}

kate_status kate_circuit_get_instruction(const kate_circuit* c, int i, int* kind, int* qbits, int* nq) {
    REQUIRE(c && kind && qbits && nq, "null pointer");
    REQUIRE(i >= 0 && i < (int)c->prog.instructions.size(), "instruction index out of range");
    auto& ins = c->prog.instructions[i];
    REQUIRE(ins.second.size() <= 256, "instruction too long for the 256-entry buffer");
    *kind = ins.first;
    *nq = (int)ins.second.size();
    for (size_t k = 0; k < ins.second.size(); k++) qbits[k] = ins.second[k];
    return KATE_OK;
}

kate_status kate_circuit_get_permutations(const kate_circuit* c, int* initial, int* final_inverse, int* valid) {
    REQUIRE(c && valid, "null pointer");
    const auto& p = c->prog;
    *valid = (int)(p.initial_permutation.size() == (size_t)p.nqbits);
    if (*valid) {
        REQUIRE(initial && final_inverse, "null permutation buffer");
        for (int i = 0; i < p.nqbits; i++) {
            initial[i] = p.initial_permutation[i];
            final_inverse[i] = p.final_inverse_permutation[i];
        }
    }
    return KATE_OK;
}

kate_status kate_merge_gates(const kate_circuit* c, int begin, int end, int* out_qbits, int* k, double* out_mat) {
    return guarded([&] {
        REQUIRE(c && out_qbits && k && out_mat, "null pointer");
        REQUIRE(begin >= 0 && end <= (int)c->prog.gates.size() && begin < end, "bad gate range");
        std::vector<kate::Gate> block(c->prog.gates.begin() + begin, c->prog.gates.begin() + end);
        kate::Gate g;
        std::string e = kate::merge_gates(block, &g);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        *k = (int)g.qbits.size();
        for (int i = 0; i < *k; i++) out_qbits[i] = g.qbits[i];
        for (size_t i = 0; i < g.dense.size(); i++) {
            out_mat[2 * i] = g.dense[i].re;
            out_mat[2 * i + 1] = g.dense[i].im;
        }
        return KATE_OK;
    });
}

namespace {
// The device merger as pass_fuse's block merger; ctx points at the device
// ordinal. Merges run on the device's default stream.
struct DeviceMergeCtx {
    int device;
};
std::string device_block_merger(const std::vector<std::vector<kate::Gate>>& blocks, void* ctx,
                                std::vector<kate::Gate>* out) {
    return kate::merge_gates_device(blocks, static_cast<DeviceMergeCtx*>(ctx)->device, nullptr, out);
}
int device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
}  // namespace

kate_status kate_merge_gates_device(const kate_circuit* c, int begin, int end, int device, void* stream,
                                    int* out_qbits, int* k, double* out_mat) {
    return guarded([&] {
        REQUIRE(c && out_qbits && k && out_mat, "null pointer");
        REQUIRE(begin >= 0 && end <= (int)c->prog.gates.size() && begin < end, "bad gate range");
        REQUIRE(device >= 0 && device < device_count(), "no such CUDA device");
        std::vector<std::vector<kate::Gate>> blocks(1);
        blocks[0].assign(c->prog.gates.begin() + begin, c->prog.gates.begin() + end);
        std::vector<kate::Gate> merged;
        std::string e = kate::merge_gates_device(blocks, device, static_cast<cudaStream_t>(stream), &merged);
        if (!e.empty()) return fail(e.rfind("cuda", 0) == 0 ? KATE_ECUDA : KATE_EINVAL, e);
        const kate::Gate& g = merged[0];
        *k = (int)g.qbits.size();
        for (int i = 0; i < *k; i++) out_qbits[i] = g.qbits[i];
        for (size_t i = 0; i < g.dense.size(); i++) {
            out_mat[2 * i] = g.dense[i].re;
            out_mat[2 * i + 1] = g.dense[i].im;
        }
        return KATE_OK;
    });
}

kate_status kate_circuit_fuse_device(kate_circuit* c, int k, double mtm, int device) {
    return guarded([&] {
        REQUIRE(c, "null circuit");
        REQUIRE(k >= 1, "qbitsizelimit must be >= 1");
        REQUIRE(device >= 0 && device < device_count(), "no such CUDA device");
        kate::Program tmp = c->prog;
        DeviceMergeCtx ctx{device};
        std::string e = kate::pass_fuse(tmp, k, mtm, device_block_merger, &ctx);
        if (!e.empty()) return fail(e.rfind("cuda", 0) == 0 ? KATE_ECUDA : KATE_EINVAL, e);
        c->prog = std::move(tmp);
        return KATE_OK;
    });
}

kate_status kate_circuit_export_qcx(const kate_circuit* c, const char* path) {
    return guarded([&] {
        REQUIRE(c && path, "null pointer");
        return from_msg(kate::export_qcx(c->prog, path));
    });
}

kate_status kate_sim_create(const kate_circuit* c, int precision, int device, kate_sim** out) {
    return guarded([&] {
        REQUIRE(c && out, "null pointer");
        REQUIRE(precision == KATE_C128 || precision == KATE_C64, "unknown precision");
        kate::Simulator* s = nullptr;
        std::string e = kate::Simulator::create(c->prog, precision, device, &s);
        if (!e.empty()) return sim_status(e);
        auto* h = new kate_sim();
        h->sim = s;
        *out = h;
        return KATE_OK;
    });
}

kate_status kate_sim_destroy(kate_sim* s) {
    if (s) {
        delete s->sim;
        delete s;
    }
    return KATE_OK;
}

kate_status kate_sim_execute(kate_sim* s, double* theta_phi) {
    return guarded([&] {
        REQUIRE(s, "null simulator");
        std::string e = s->sim->run_async(nullptr, nullptr);
        if (e.empty()) e = s->sim->synchronize();
        if (e.empty() && theta_phi) e = s->sim->proba_state(theta_phi);
        return sim_status(e);
    });
}

kate_status kate_sim_execute_from(kate_sim* s, const double* in, double* out) {
    return guarded([&] {
        REQUIRE(s && in, "null pointer");
        std::string e = s->sim->run_async(nullptr, in);
        if (e.empty()) e = s->sim->synchronize();
        if (e.empty() && out) e = s->sim->proba_state(out);
        return sim_status(e);
    });
}

kate_status kate_sim_execute_timed(kate_sim* s, const double* in, double* out, double* ms) {
    return guarded([&] {
        REQUIRE(s, "null simulator");
        return sim_status(s->sim->execute_timed(in, out, ms));
    });
}

kate_status kate_sim_run_async(kate_sim* s, void* stream) {
    return guarded([&] {
        REQUIRE(s, "null simulator");
        return sim_status(s->sim->run_async(stream, nullptr));
    });
}

kate_status kate_sim_synchronize(kate_sim* s) {
    REQUIRE(s, "null simulator");
    return sim_status(s->sim->synchronize());
}

kate_status kate_sim_proba_state(kate_sim* s, double* tp) {
    return guarded([&] {
        REQUIRE(s && tp, "null pointer");
        return sim_status(s->sim->proba_state(tp));
    });
}

kate_status kate_sim_get_state(kate_sim* s, double* out) {
    return guarded([&] {
        REQUIRE(s && out, "null pointer");
        return sim_status(s->sim->get_state(out));
    });
}

kate_status kate_sim_set_state(kate_sim* s, const double* in) {
    return guarded([&] {
        REQUIRE(s && in, "null pointer");
        return sim_status(s->sim->set_state(in));
    });
}

kate_status kate_sim_expect_z(kate_sim* s, double* out) {
    return guarded([&] {
        REQUIRE(s && out, "null pointer");
        return sim_status(s->sim->expect_z(out));
    });
}

kate_status kate_sim_probabilities(kate_sim* s, double* out) {
    return guarded([&] {
        REQUIRE(s && out, "null pointer");
        return sim_status(s->sim->probabilities(out));
    });
}

kate_status kate_sim_sample(kate_sim* s, int shots, uint64_t seed, uint64_t* out) {
    return guarded([&] {
        REQUIRE(s && (out || shots == 0), "null pointer");
        return sim_status(s->sim->sample(shots, seed, out));
    });
}

kate_status kate_sim_state_device(kate_sim* s, void** dptr, int* phys) {
    REQUIRE(s && dptr && phys, "null pointer");
    return sim_status(s->sim->state_device(dptr, phys));
}

kate_status kate_sim_profile_passes(kate_sim* s, float* ms, float* init_ms) {
    return guarded([&] {
        REQUIRE(s && ms, "null pointer");
        return sim_status(s->sim->profile_passes(ms, init_ms));
    });
}

kate_status kate_sim_launches_per_run(kate_sim* s, int* out) {
    REQUIRE(s && out, "null pointer");
    *out = s->sim->launches_per_run();
    return KATE_OK;
}

kate_status kate_sim_norm2_before_renorm(kate_sim* s, double* norm2) {
    REQUIRE(s && norm2, "null pointer");
    const std::string e = s->sim->norm2_before_renorm(norm2);
    if (e.rfind("no run", 0) == 0) return fail(KATE_ESTATE, e);
    if (!e.empty()) return fail(e.find("complex64") != std::string::npos ? KATE_EINVAL : KATE_ECUDA, e);
    return KATE_OK;
}

kate_status kate_sim_pass_kernel(kate_sim* s, int i, int* kind) {
    REQUIRE(s && kind, "null pointer");
    const int k = s->sim->pass_kernel(i);
    REQUIRE(k >= 0, "pass index out of range");
    *kind = k;
    return KATE_OK;
}

kate_status kate_sim_pass_work(kate_sim* s, int i, double* out3) {
    REQUIRE(s && out3, "null pointer");
    REQUIRE(s->sim->pass_kernel(i) >= 0, "pass index out of range");
    if (!s->sim->pass_work(i, out3)) return fail(KATE_EINVAL, "pass is not run by a pass-specialised kernel");
    return KATE_OK;
}

kate_status kate_sim_nqbits(kate_sim* s, int* out) {
    REQUIRE(s && out, "null pointer");
    *out = s->sim->nqbits();
    return KATE_OK;
}

kate_status kate_sim_num_passes(kate_sim* s, int* out) {
    REQUIRE(s && out, "null pointer");
    *out = (int)s->sim->plan().passes.size();
    return KATE_OK;
}

kate_status kate_sim_get_pass(kate_sim* s, int i, int* tile_qbits, int* m, int* ngates) {
    REQUIRE(s && tile_qbits && m && ngates, "null pointer");
    const auto& P = s->sim->plan();
    REQUIRE(i >= 0 && i < (int)P.passes.size(), "pass index out of range");
    const auto& p = P.passes[i];
    *m = (int)p.tile.size();
    for (size_t k = 0; k < p.tile.size(); k++) tile_qbits[k] = p.tile[k];
    *ngates = (int)p.gates.size();
    return KATE_OK;
}

kate_status kate_plan_create(const kate_circuit* c, int max_tile, int coalesce, unsigned flags, kate_plan** out) {
    return guarded([&] {
        REQUIRE(c && out, "null pointer");
        REQUIRE(max_tile >= 1 && max_tile <= KATE_MAX_TILE, "max_tile must be in [1, 14]");
        REQUIRE(coalesce >= 0 && coalesce <= max_tile, "coalesce must be in [0, max_tile]");
        kate::Program prog = c->prog;
        if (prog.instructions.empty()) {
            std::string e = kate::pass_compile_default(prog, 0, prog.nqbits);
            if (!e.empty()) return fail(KATE_EINVAL, e);
        }
        kate::PlanOptions opt;
        opt.max_tile = max_tile;
        opt.coalesce = coalesce;
        opt.remap = !(flags & KATE_PLAN_NO_REMAP);
        opt.remap_search = (flags & KATE_PLAN_REMAP_SEARCH) != 0;
        opt.cap_search = opt.remap_search;
        opt.fuse_1q = !(flags & KATE_PLAN_NO_FUSE1Q);
        opt.c64 = (flags & KATE_PLAN_C64) != 0;
        opt.dense2_reg = !opt.c64 && !(flags & KATE_PLAN_NO_DENSE2);
        auto* p = new kate_plan();
        std::string e = kate::build_plan(prog, opt, &p->plan);
        if (!e.empty()) {
            delete p;
            return fail(KATE_EINVAL, e);
        }
        for (auto& pp : p->plan.passes) {
            p->passes.push_back(kate::to_devpass(prog.nqbits, pp, (int)p->ops.size()));
            p->ops.insert(p->ops.end(), pp.ops.begin(), pp.ops.end());
        }
        *out = p;
        return KATE_OK;
    });
}

kate_status kate_plan_destroy(kate_plan* p) {
    delete p;
    return KATE_OK;
}

kate_status kate_plan_num_passes(const kate_plan* p, int* out) {
    REQUIRE(p && out, "null pointer");
    *out = (int)p->passes.size();
    return KATE_OK;
}

kate_status kate_plan_get_pass(const kate_plan* p, int i, int* info, uint8_t* tphys, uint8_t* outsrc) {
    REQUIRE(p && info && tphys && outsrc, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->passes.size(), "pass index out of range");
    const DevPass& d = p->passes[i];
    info[0] = d.m;
    info[1] = d.nops;
    info[2] = d.op0;
    info[3] = d.ncb;
    for (int t = 0; t < 16; t++) {
        tphys[t] = d.tphys[t];
        outsrc[t] = d.outsrc[t];
    }
    return KATE_OK;
}

kate_status kate_plan_num_ops(const kate_plan* p, int* out) {
    REQUIRE(p && out, "null pointer");
    *out = (int)p->ops.size();
    return KATE_OK;
}

namespace {
kate_status export_op(const kate::Plan& plan, const DevOp& o, int* ints, uint64_t* pmask, double* vals) {
    ints[0] = o.kind;
    ints[1] = o.k;
    for (int j = 0; j < 5; j++) {
        ints[2 + j] = o.tb[j];
        ints[7 + j] = o.ftb[j];
        ints[12 + j] = o.fpos[j];
    }
    ints[17] = (int)o.tmask;
    *pmask = o.pmask;
    vals[0] = o.ph_re;
    vals[1] = o.ph_im;
    size_t len = 0;
    if (o.kind == OPK_DENSE) len = (size_t)1 << (2 * o.k);
    else if (o.kind == OPK_DIAG) len = (size_t)1 << o.k;
    for (size_t j = 0; j < len; j++) {
        vals[2 + 2 * j] = plan.pool[o.mat + j].re;
        vals[3 + 2 * j] = plan.pool[o.mat + j].im;
    }
    return KATE_OK;
}
}  // namespace

kate_status kate_plan_get_op(const kate_plan* p, int i, int* ints, uint64_t* pmask, double* vals) {
    REQUIRE(p && ints && pmask && vals, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->ops.size(), "op index out of range");
    return export_op(p->plan, p->ops[i], ints, pmask, vals);
}

kate_status kate_plan_get_program(const kate_plan* p, int i, void* out, size_t cap, size_t* size, int* has) {
    REQUIRE(p && size && has, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->plan.passes.size(), "pass index out of range");
    *size = sizeof(PassProg);
    const auto& pp = p->plan.passes[i];
    *has = pp.prog ? 1 : 0;
    if (pp.prog && out && cap >= sizeof(PassProg)) std::memcpy(out, pp.prog.get(), sizeof(PassProg));
    return KATE_OK;
}

kate_status kate_plan_pass_source(const kate_plan* p, int i, int from_zero, char* out, size_t cap, size_t* size) {
    REQUIRE(p && size, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->plan.passes.size(), "pass index out of range");
    const auto& pp = p->plan.passes[i];
    REQUIRE(pp.prog != nullptr, "pass has no register-staged program");
    std::string why;
    REQUIRE(from_zero >= 0 && from_zero <= 2, "from_zero must be 0, 1 or 2");
    const std::string src = kate::jit_pass_source(*pp.prog, &why, from_zero);
    REQUIRE(!src.empty(), "pass has no specialised kernel: " + why);
    *size = src.size() + 1;
    if (out && cap >= src.size() + 1) std::memcpy(out, src.c_str(), src.size() + 1);
    return KATE_OK;
}

kate_status kate_plan_get_block_program(const kate_plan* p, int i, void* out, size_t cap, size_t* size, int* has) {
    REQUIRE(p && size && has, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->plan.passes.size(), "pass index out of range");
    *size = sizeof(BlockProg);
    const auto& pp = p->plan.passes[i];
    *has = pp.bprog ? 1 : 0;
    if (pp.bprog && out && cap >= sizeof(BlockProg)) std::memcpy(out, pp.bprog.get(), sizeof(BlockProg));
    return KATE_OK;
}

kate_status kate_plan_block_images(const kate_plan* p, void* out, size_t cap, size_t* size) {
    REQUIRE(p && size, "null pointer");
    *size = p->plan.bimg.size();
    if (out && cap >= p->plan.bimg.size()) std::memcpy(out, p->plan.bimg.data(), p->plan.bimg.size());
    return KATE_OK;
}

kate_status kate_plan_num_smem_ops(const kate_plan* p, int* out) {
    REQUIRE(p && out, "null pointer");
    *out = (int)p->plan.smem_ops.size();
    return KATE_OK;
}

kate_status kate_plan_get_smem_op(const kate_plan* p, int i, int* ints, uint64_t* pmask, double* vals) {
    REQUIRE(p && ints && pmask && vals, "null pointer");
    REQUIRE(i >= 0 && i < (int)p->plan.smem_ops.size(), "op index out of range");
    return export_op(p->plan, p->plan.smem_ops[i], ints, pmask, vals);
}

kate_status kate_plan_final_layout(const kate_plan* p, int* phys, int* l2l) {
    REQUIRE(p && phys && l2l, "null pointer");
    for (int q = 0; q < p->plan.n; q++) {
        phys[q] = p->plan.final_phys[q];
        l2l[q] = p->plan.label_to_logical[q];
    }
    return KATE_OK;
}

// ---- batches ----

namespace {
kate::BatchOptions to_options(const kate_batch_options* o) {
    kate::BatchOptions r;
    if (!o) return r;
    if (o->chunk > 0) r.chunk = o->chunk;
    if (o->zchunks > 0) r.zchunks = o->zchunks;
    r.window_bytes = o->window_bytes;
    if (o->wait_ms > 0) r.wait_ms = o->wait_ms;
    r.fault_task = o->fault_task > 0 ? o->fault_task - 1 : -1;
    r.tune.resize(KATE_BATCH_MAX_QUBITS + 1);
    for (int n = 0; n <= KATE_BATCH_MAX_QUBITS; n++) {
        // A field left at 0 takes its default, each on its own (so a caller
        // can set one choice, e.g. blocks, and leave the rest).
        r.tune[n].fusion = o->tune[n].fusion > 0 ? o->tune[n].fusion : 1;
        r.tune[n].max_gates = o->tune[n].max_gates > 0 ? o->tune[n].max_gates : 96;
        r.tune[n].group = o->tune[n].group_qubits > 0 ? o->tune[n].group_qubits : KATE_TILE_BITS;
        r.tune[n].coalesce = o->tune[n].coalesce > 0 ? o->tune[n].coalesce : 4;
        r.tune[n].blocks = o->tune[n].blocks ? 1 : 0;
    }
    return r;
}

std::vector<const kate::Program*> programs(const kate_circuit* const* c, int count) {
    std::vector<const kate::Program*> v;
    for (int i = 0; i < count; i++) v.push_back(c[i] ? &c[i]->prog : nullptr);
    return v;
}
}  // namespace

kate_status kate_release_cached_memory(int device) {
    return guarded([&] {
        kate::release_cached(device);
        return KATE_OK;
    });
}

kate_status kate_batch_options_default(kate_batch_options* opt) {
    REQUIRE(opt, "null pointer");
    std::memset(opt, 0, sizeof(*opt));
    kate::BatchOptions d;
    opt->chunk = d.chunk;
    opt->zchunks = d.zchunks;
    opt->wait_ms = d.wait_ms;
    return KATE_OK;
}

kate_status kate_batch_autotune(const kate_circuit* const* circuits, int count, int precision, int device,
                                kate_batch_options* opt) {
    return guarded([&] {
        REQUIRE(circuits && opt && count > 0, "null pointer or empty batch");
        REQUIRE(precision == KATE_C128 || precision == KATE_C64, "unknown precision");
        for (int i = 0; i < count; i++) REQUIRE(circuits[i], "null circuit");
        kate::BatchOptions o = to_options(opt);
        std::string e = kate::batch_autotune(programs(circuits, count), precision, device, &o);
        if (!e.empty()) return sim_status(e);
        for (int n = 0; n <= KATE_BATCH_MAX_QUBITS; n++) {
            opt->tune[n].fusion = o.tune[n].fusion;
            opt->tune[n].max_gates = o.tune[n].max_gates;
            opt->tune[n].group_qubits = o.tune[n].group;
            opt->tune[n].coalesce = o.tune[n].coalesce;
            opt->tune[n].blocks = o.tune[n].blocks;
        }
        return KATE_OK;
    });
}

kate_status kate_batch_create(const kate_circuit* const* circuits, int count, int precision, int device,
                              const kate_batch_options* opt, kate_batch** out) {
    return guarded([&] {
        REQUIRE(circuits && out && count > 0, "null pointer or empty batch");
        REQUIRE(precision == KATE_C128 || precision == KATE_C64, "unknown precision");
        for (int i = 0; i < count; i++) REQUIRE(circuits[i], "null circuit");
        kate::Batch* b = nullptr;
        std::string e = kate::Batch::create(programs(circuits, count), precision, device, to_options(opt), &b);
        if (!e.empty()) return sim_status(e);
        auto* h = new kate_batch();
        h->b = b;
        h->ncirc = count;
        *out = h;
        return KATE_OK;
    });
}

kate_status kate_batch_destroy(kate_batch* b) {
    if (b) {
        delete b->b;
        delete b;
    }
    return KATE_OK;
}

kate_status kate_batch_run_async(kate_batch* b, void* stream) {
    return guarded([&] {
        REQUIRE(b, "null batch");
        return sim_status(b->b->run_async(stream));
    });
}

kate_status kate_batch_synchronize(kate_batch* b) {
    return guarded([&] {
        REQUIRE(b, "null batch");
        std::string e = b->b->synchronize();
        if (!e.empty()) return device_status(e);
        return KATE_OK;
    });
}

kate_status kate_batch_run(kate_batch* b) {
    return guarded([&] {
        REQUIRE(b, "null batch");
        std::string e = b->b->run_async(nullptr);
        if (!e.empty()) return sim_status(e);
        e = b->b->synchronize();
        if (!e.empty()) return device_status(e);
        return KATE_OK;
    });
}

kate_status kate_batch_expect_z(kate_batch* b, double* out) {
    return guarded([&] {
        REQUIRE(b && out, "null pointer");
        std::string e = b->b->expect_z(out);
        if (!e.empty()) return device_status(e);
        return KATE_OK;
    });
}

kate_status kate_batch_num_outputs(const kate_batch* b, long long* out) {
    REQUIRE(b && out, "null pointer");
    *out = (long long)b->b->num_outputs();
    return KATE_OK;
}

kate_status kate_batch_info(const kate_batch* b, long long* info) {
    REQUIRE(b && info, "null pointer");
    info[0] = (long long)b->b->num_tasks();
    info[1] = (long long)b->b->num_programs();
    info[2] = (long long)b->b->arena_bytes();
    info[3] = (long long)b->b->grid();
    return KATE_OK;
}

kate_status kate_batch_block_programs(const kate_batch* b, long long* out) {
    REQUIRE(b && out, "null pointer");
    *out = (long long)b->b->num_block_programs();
    return KATE_OK;
}

kate_status kate_batch_create_times(const kate_batch* b, double* ms) {
    REQUIRE(b && ms, "null pointer");
    b->b->create_times(ms);
    return KATE_OK;
}

kate_status kate_batch_upload_bytes(const kate_batch* b, long long* bytes) {
    REQUIRE(b && bytes, "null pointer");
    *bytes = (long long)b->b->upload_bytes();
    return KATE_OK;
}

kate_status kate_batch_circuit_info(const kate_batch* b, int* programs, int* resident_qubits) {
    REQUIRE(b && programs && resident_qubits, "null pointer");
    for (int i = 0; i < b->ncirc; i++) b->b->circuit_info(i, programs + i, resident_qubits + i);
    return KATE_OK;
}

kate_status kate_batch_get_state(kate_batch* b, int circuit, double* out) {
    return guarded([&] {
        REQUIRE(b && out, "null pointer");
        std::string e = b->b->get_state(circuit, out);
        if (e.find("no resident state") != std::string::npos || e.find("out of range") != std::string::npos)
            return fail(KATE_EINVAL, e);
        if (!e.empty()) return device_status(e);
        return KATE_OK;
    });
}

kate_status kate_batch_time(kate_batch* b, int runs, float* ms) {
    return guarded([&] {
        REQUIRE(b && ms && runs > 0, "null pointer or no runs");
        std::string e = b->b->time_runs(runs, ms);
        if (!e.empty()) return device_status(e);
        return KATE_OK;
    });
}

// ---- serving ----

kate_status kate_server_options_default(kate_server_options* opt) {
    REQUIRE(opt, "null pointer");
    std::memset(opt, 0, sizeof(*opt));
    kate::ServeOptions d;
    opt->budget_bytes = d.budget_bytes;
    opt->aux_bytes = d.aux_bytes;
    opt->step_tiles = d.step_tiles;
    opt->chunk = d.chunk;
    opt->zchunks = d.zchunks;
    opt->schunks = d.schunks;
    opt->planners = d.planners;
    opt->fusion = d.tune.fusion;
    opt->max_gates = d.tune.max_gates;
    opt->step_latency_us = d.step_latency_us;
    opt->tensor_blocks = d.tune.blocks;
    return KATE_OK;
}

kate_status kate_server_create(int precision, int device, const kate_server_options* opt, kate_server** out) {
    return guarded([&] {
        REQUIRE(out, "null pointer");
        REQUIRE(precision == KATE_C128 || precision == KATE_C64, "unknown precision");
        kate::ServeOptions o;
        if (opt) {
            if (opt->budget_bytes) o.budget_bytes = opt->budget_bytes;
            if (opt->aux_bytes) o.aux_bytes = opt->aux_bytes;
            if (opt->step_tiles > 0) o.step_tiles = opt->step_tiles;
            if (opt->chunk > 0) o.chunk = opt->chunk;
            if (opt->zchunks > 0) o.zchunks = opt->zchunks;
            if (opt->schunks > 0) o.schunks = opt->schunks;
            o.planners = opt->planners;
            if (opt->fusion > 0) o.tune.fusion = opt->fusion;
            if (opt->max_gates > 0) o.tune.max_gates = opt->max_gates;
            if (opt->step_latency_us > 0) o.step_latency_us = opt->step_latency_us;
            if (opt->step_latency_us < 0) o.step_latency_us = 0;
            o.tune.blocks = opt->tensor_blocks ? 1 : 0;
        }
        kate::Server* s = nullptr;
        std::string e = kate::Server::create(precision, device, o, &s);
        if (!e.empty()) return sim_status(e);
        auto* h = new kate_server();
        h->s = s;
        *out = h;
        return KATE_OK;
    });
}

kate_status kate_server_destroy(kate_server* s) {
    if (s) {
        delete s->s;
        delete s;
    }
    return KATE_OK;
}

kate_status kate_server_submit(kate_server* s, const kate_circuit* c, int shots, uint64_t seed, long long* id) {
    return guarded([&] {
        REQUIRE(s && c && id, "null pointer");
        int64_t v = 0;
        std::string e = s->s->submit(c->prog, shots, seed, &v);
        if (!e.empty()) return fail(KATE_EINVAL, e);
        *id = (long long)v;
        return KATE_OK;
    });
}

kate_status kate_server_wait(kate_server* s, long long id, double timeout_s, int* nqbits, double* z,
                             uint64_t* samples, double* times) {
    return guarded([&] {
        REQUIRE(s, "null server");
        kate::ServeResult r;
        std::string e = s->s->wait(id, timeout_s, &r);
        if (e == "timeout") return fail(KATE_ETIMEDOUT, "request not finished within the timeout");
        if (!e.empty()) return sim_status(e);
        if (nqbits) *nqbits = r.n;
        if (z) std::memcpy(z, r.z.data(), r.z.size() * sizeof(double));
        if (samples && !r.samples.empty()) std::memcpy(samples, r.samples.data(), r.samples.size() * sizeof(uint64_t));
        if (times) {
            times[0] = r.t_submit;
            times[1] = r.t_admit;
            times[2] = r.t_done;
        }
        return KATE_OK;
    });
}

kate_status kate_server_stats(const kate_server* s, long long* out) {
    REQUIRE(s && out, "null pointer");
    int64_t v[12];
    s->s->stats(v);
    for (int i = 0; i < 12; i++) out[i] = (long long)v[i];
    return KATE_OK;
}

kate_status kate_server_now(const kate_server* s, double* t) {
    REQUIRE(s && t, "null pointer");
    *t = s->s->now();
    return KATE_OK;
}

}  // extern "C"
