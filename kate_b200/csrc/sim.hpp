// Device simulator: owns the state vector and runs planned group passes.
// Replaces the reference's GPU Simulator (HIPcode/simulator.hpp:220-811).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "plan.hpp"

namespace kate {

struct SimImpl;

class Simulator {
public:
    // Copies `prog` (compiling it with compileDefault(0) when it has no
    // instructions), plans the passes and allocates the state on `device`.
    static std::string create(const Program& prog, int precision, int device, Simulator** out);
    ~Simulator();

    std::string run_async(void* stream, const double* theta_phi_in);  // init + all passes, no sync
    std::string synchronize();
    // init + passes with CUDA events between them, then the measurement on
    // the host clock: ms[0] init, ms[1] group passes, ms[2] proba_state,
    // ms[3] number of passes. tp_in / tp_out nullable.
    std::string execute_timed(const double* tp_in, double* tp_out, double* ms);
    std::string proba_state(double* theta_phi);                       // reference measurement
    std::string get_state(double* out);                               // 2*2^n doubles, label order
    std::string set_state(const double* in);
    std::string expect_z(double* out);
    std::string probabilities(double* out);
    std::string sample(int shots, uint64_t seed, uint64_t* out);
    std::string state_device(void** dptr, int* phys);
    std::string profile_passes(float* ms, float* init_ms);
    int launches_per_run() const;
    // Kernel that runs pass i: 0 generic shared-memory kernel, 1 register-
    // staged interpreter, 2 pass-specialised kernel, 3 complex64 tensor-core
    // blocks; -1 for an index out of range.
    int pass_kernel(int i) const;
    // Work per amplitude of pass i when a pass-specialised kernel runs it:
    // out = {HBM bytes, FP64 instructions, shared-memory bytes}; false for
    // other kernels.
    bool pass_work(int i, double out[3]) const;
    // Complex64: ||psi||^2 of the last run's state before it was rescaled to
    // norm 1 (FP64 reduction on the device).
    std::string norm2_before_renorm(double* out);

    int nqbits() const;
    int precision() const;
    const Plan& plan() const;
    SimImpl* impl() { return d_; }

private:
    // Queue the initial state / every group pass on stream st (cudaStream_t).
    std::string enqueue_init(void* st, const double* tp);
    std::string enqueue_passes(void* st);
    SimImpl* d_ = nullptr;
};

}  // namespace kate
