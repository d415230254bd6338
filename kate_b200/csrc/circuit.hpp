// Circuit IR and the host-side compile passes.
//
// The passes reproduce the reference's decisions exactly (same schedules,
// same fusion intervals, same groups, same permutations), because the gate
// list they produce is part of the drop-in contract: a user who runs
// gateScheduling + gateFusion + gateGrouping gets the same compiled program
// as with the reference. The code is this project's own; the algorithms are
// the reference's (backendagnosticcode/Circuit.hpp, QuantumCircuit.hpp,
// graphUtil.hpp, CPUcode/GateMerger.hpp).
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace kate {

// Gate identifiers (backendagnosticcode/agnosticpreprocessor.hpp:28-33).
enum GateId : int { G_DENSE = 0, G_H = 2, G_CNOT = 3, G_CRK = 4, G_TOFFOLI = 5, G_RX = 6, G_RZ = 7 };

// Complex double with the reference's exact operation order
// (backendagnosticcode/basic_host_types.hpp:34-78), so merged matrices are
// bit-identical to the reference's CPU merger.
struct Cx {
    double re = 0.0, im = 0.0;
    Cx() = default;
    Cx(double r, double i) : re(r), im(i) {}
};
inline Cx operator+(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx operator-(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx operator*(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx operator*(Cx a, double d) { return {a.re * d, a.im * d}; }

struct Gate {
    int id = -1;
    std::vector<int> qbits;
    int optarg = 0;
    std::vector<Cx> dense;  // row-major 2^k x 2^k when id == G_DENSE
};

struct Program {
    int nqbits = 0;
    std::vector<Gate> gates;                                     // gate_set_ordered
    std::vector<std::pair<int, std::vector<int>>> groups;        // (end index, sorted qubit set)
    std::vector<int> initial_permutation;                        // real -> virtual
    std::vector<int> final_inverse_permutation;                  // virtual -> real
    std::vector<std::pair<int, std::vector<int>>> instructions;  // (0, swap pairs) | (1, {})
};

// Every pass returns "" on success, or an error message (the program is then
// left unchanged).
std::string validate_gate(const Program& p, const Gate& g);
std::string pass_schedule(Program& p);
// Merges every block of gates into one dense gate each (out[b] for
// blocks[b]); "" on success. pass_fuse takes one to run all of its merges in
// one call (the device merger); without one it merges on the host.
using BlockMerger = std::string (*)(const std::vector<std::vector<Gate>>& blocks, void* ctx, std::vector<Gate>* out);
std::string pass_fuse(Program& p, int qbitsizelimit, double merge_time_matters, BlockMerger merger = nullptr,
                      void* ctx = nullptr);
std::string pass_group(Program& p, int qbitgroupsize);
std::string pass_allocate(Program& p, int numberofgpulog2, int maxlocalqbitnumber);
std::string pass_compile_default(Program& p, int numberofgpulog2, int maxlocalqbitnumber);
std::string export_qcx(const Program& p, const std::string& path);

// FP64 product of `gates` as one dense gate on the sorted union of their
// qubits (CPUcode/GateMerger.hpp:8-55). k must be <= 10.
std::string merge_gates(const std::vector<Gate>& gates, Gate* out);

// Applies one gate to a 2^k local state whose bit i is qubit local[i]
// position; used by the merger (CPUcode/GateComputing.hpp:6-129 arithmetic).
void apply_gate_local(const Gate& g, const int* local_bits, int k, Cx* state);

}  // namespace kate
