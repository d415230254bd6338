// Test and measurement infrastructure only: a C-ABI harness around the
// reference simulator's own GPU path (Line-fr/Kate built with nvcc, which
// selects HIPcode/* through HIPcode/HIPpreprocessor.hpp). It is compiled from
// the reference headers where they lie (oracle/Makefile, target refgpu) into
// oracle/_ref/, never copied. Nothing in the product links or loads it; only
// the GPU tests and bench.py's reference-GPU leg do.
//
// Reference entry points driven here (paths within the reference project):
//   Circuit / appendGate / Gate        backendagnosticcode/QuantumCircuit.hpp:18-37,
//                                      backendagnosticcode/basic_host_types.hpp:198-245
//   gateScheduling/gateFusion/gateGrouping
//                                      backendagnosticcode/Circuit.hpp:12-206
//   compileDefault                     backendagnosticcode/QuantumCircuit.hpp:126-204
//   Simulator (GPU) ctor               HIPcode/simulator.hpp:243-300
//   initialize / executeCommand        HIPcode/simulator.hpp:427-443, 760-810
//   measurement -> proba_state         HIPcode/simulator.hpp:483-543
//
// Safety limit. executeCommand gives the group kernel sharedMemPerBlock/4
// bytes of dynamic shared memory (12 KiB on this GPU) and cancels a group only
// when 2^qubits exceeds that number of BYTES (HIPcode/simulator.hpp:785-793),
// so groups of 10..13 qubits would read and write past the 12 KiB. With at
// most 9 qubits per group the state tile is 8 KiB, a dense gate of <= 4 qubits
// is staged in the remaining 4 KiB (HIPcode/GPUGate.hpp:153-166, size checked
// in bytes there) and a 5-qubit one is read from global memory; with one
// thread per amplitude every thread runs exactly one (line, row) iteration,
// so the __syncthreads inside the dense loop (HIPcode/GPUGate.hpp:196) is
// reached by all threads. krefg_session_new therefore refuses circuits with a
// group above 9 qubits, a gate above 5 qubits, or a swap instruction.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits.h>
#include <list>
#include <math.h>
#include <queue>
#include <set>
#include <stdlib.h>
#include <string>
#include <thread>
#include <vector>
#define private public
#include "Kate.hpp"
#undef private

#include <cuda_runtime.h>

namespace {

constexpr int MAX_GROUP_QUBITS = 9;
constexpr int MAX_GATE_QUBITS = 5;

struct Handle {
    Kate::Circuit circ;
    explicit Handle(int n) : circ(n) {}
};

Kate::Gate make_gate(int id, int nq, const int* qbits, int optarg, const double* dense) {
    std::vector<int> q(qbits, qbits + nq);
    if (id == 0) {
        int dim = 1 << nq;
        Kate::Matrix<Kate::Complex> m(dim);
        for (int i = 0; i < dim * dim; i++) m.data[i] = Kate::Complex(dense[2 * i], dense[2 * i + 1]);
        return Kate::Gate(m, q);
    }
    return Kate::Gate(id, q, optarg);
}

int last_cuda_error() {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e;
}

}  // namespace

extern "C" {

void* krefg_circuit_new(int n) { return new Handle(n); }
void krefg_free(void* h) { delete static_cast<Handle*>(h); }

void krefg_append(void* h, int id, int nq, const int* qbits, int optarg, const double* dense) {
    static_cast<Handle*>(h)->circ.appendGate(make_gate(id, nq, qbits, optarg, dense));
}

void krefg_schedule(void* h) { static_cast<Handle*>(h)->circ.gateScheduling(); }
void krefg_fuse(void* h, int k, double mtm) { static_cast<Handle*>(h)->circ.gateFusion(k, mtm); }
void krefg_group(void* h, int m) { static_cast<Handle*>(h)->circ.gateGrouping(m); }
void krefg_compile_default(void* h, int g, int maxlocal) {
    static_cast<Handle*>(h)->circ.compileDefault(g, maxlocal);
}

int krefg_ngates(void* h) { return (int)static_cast<Handle*>(h)->circ.gate_set_ordered.size(); }
int krefg_ngroups(void* h) { return (int)static_cast<Handle*>(h)->circ.groups.size(); }

// Largest group, in qubits, of the compiled circuit (0 when not grouped).
int krefg_max_group(void* h) {
    size_t m = 0;
    for (auto& g : static_cast<Handle*>(h)->circ.groups) m = std::max(m, g.second.size());
    return (int)m;
}

// Why krefg_session_new would refuse the circuit: 0 = accepted, 1 = not
// compiled, 2 = a group above 9 qubits, 3 = a gate above 5 qubits, 4 = a swap
// instruction, 5 = a gate outside its group.
int krefg_check(void* h) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    if (c.instructions.empty() || c.groups.empty()) return 1;
    for (auto& g : c.groups)
        if ((int)g.second.size() > MAX_GROUP_QUBITS) return 2;
    for (auto& g : c.gate_set_ordered)
        if ((int)g.qbits.size() > MAX_GATE_QUBITS) return 3;
    for (auto& ins : c.instructions)
        if (ins.first != 1) return 4;
    size_t b = 0;
    for (auto& g : c.groups) {
        for (size_t i = b; i < (size_t)g.first && i < c.gate_set_ordered.size(); i++)
            for (int q : c.gate_set_ordered[i].qbits)
                if (!g.second.count(q)) return 5;
        b = g.first;
    }
    return 0;
}

// A GPU Simulator on the compiled circuit (device 0). Returns null when the
// circuit fails krefg_check, when no GPU is present (the reference would fall
// back to its CPU path) or when a CUDA call failed; *status receives the
// reason (krefg_check's code, 10 = no GPU, negative = CUDA error).
void* krefg_session_new(void* h, int* status) {
    Kate::Circuit& c = static_cast<Handle*>(h)->circ;
    int chk = krefg_check(h);
    if (chk != 0) {
        if (status) *status = chk;
        return nullptr;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        if (status) *status = 10;
        return nullptr;
    }
    auto* sim = new Kate::Simulator(c, 1);
    int e = last_cuda_error();
    if (sim->cpumode || e != 0) {
        delete sim;
        if (status) *status = e != 0 ? e : 10;
        return nullptr;
    }
    if (status) *status = 0;
    return sim;
}

// One gate phase: |0..0> (initialize, not timed), then every compute
// instruction through the reference's executeCommand, which synchronises the
// device after each group. *ms receives the wall time of the instruction loop.
// Returns 0 or a negative CUDA error.
int krefg_session_run(void* s, double* ms) {
    auto* sim = static_cast<Kate::Simulator*>(s);
    sim->initialize();
    int e = last_cuda_error();
    if (e != 0) return e;
    auto t0 = std::chrono::steady_clock::now();
    int groupid = 0;
    for (const auto& instr : sim->instructions) {
        if (instr.first == 1) {
            sim->executeCommand(groupid);
            groupid++;
        }
    }
    e = last_cuda_error();
    auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return e;
}

// The reference's measurement (proba_state) of the current state: 2*n
// doubles, (theta, phi) per qubit.
int krefg_session_measure(void* s, double* proba_out) {
    auto* sim = static_cast<Kate::Simulator*>(s);
    Kate::proba_state res = sim->measurement();
    for (int i = 0; i < sim->nqbits; i++) {
        proba_out[2 * i] = res.val[i].first;
        proba_out[2 * i + 1] = res.val[i].second;
    }
    return last_cuda_error();
}

// Copies the device state (2 * 2^n doubles, the simulator's amplitude order).
int krefg_session_state(void* s, double* out) {
    auto* sim = static_cast<Kate::Simulator*>(s);
    size_t bytes = sizeof(Kate::Complex) << sim->nqbits;
    cudaError_t e = cudaMemcpy(out, sim->gpu_qbits_states[0], bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -(int)e;
}

void krefg_session_free(void* s) { delete static_cast<Kate::Simulator*>(s); }

}  // extern "C"
