// Group-pass planner: turns a compiled program into B200 group passes.
//
// A group pass reads every amplitude once and writes it once. It owns a
// "tile" of m qubits: each CTA takes one coset of the tile (the 2^m
// amplitudes that share all non-tile bits), stages it on chip, applies every
// planned gate to it and writes it back. Gates are classified as
//   - target qubits: must be tile qubits (dense, H, the X of CNOT/TOFFOLI);
//   - free qubits: controls and diagonal qubits; they may lie outside the
//     tile, where they are constant over a coset and are evaluated once per
//     CTA from the coset's base address.
// The planner packs gates greedily in program order (a gate is taken when
// none of its qubits is blocked by an earlier skipped gate and its targets
// fit the tile), which is the single-GPU replacement for the reference's
// gateGrouping + per-group launches (backendagnosticcode/Circuit.hpp:176-206,
// HIPcode/simulator.hpp:760-810).
//
// Qubit remap (the replacement for the reference's swap instructions,
// HIPcode/simulator.hpp:639-759): the c lowest physical bits must be tile
// bits so that every load/store touches 2^c contiguous amplitudes. Each pass
// may write its tile back with its tile bits permuted, which moves c qubits
// that the next pass needs into those low positions at no extra HBM cost.
// Swap instructions of the compiled program become pure relabelings.
// Which c tile qubits go low decides what the next pass can take (it holds
// them and m - c more). With remap_search the planner tries every c-subset
// of the tile and keeps the one that lets the next pass take the most
// gates; otherwise it takes the first c tile qubits the next pass's greedy
// selection reaches. The pass count then depends on the gate cap per pass
// in no monotone way (a cap cuts a pass's gates to a program-order prefix,
// which changes what the next pass can reach); with cap_search the planner
// plans with each of a few caps and keeps the plan with the fewest passes
// (passes left without a register-staged program count as ten).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "device_types.h"

namespace kate {

struct PlanOptions {
    int max_tile = 12;   // tile qubits per pass (the kernels' tile)
    int group_qubits = 0;  // m: qubits the gates of one pass may span, at most max_tile (0: max_tile); the
                           // rest of the tile is filled with other qubits (the reference's gateGrouping(m))
    int coalesce = 4;    // c: low physical bits every tile must contain
    bool remap = true;   // move next-needed qubits into the low bits on write
    bool remap_search = false;  // choose those qubits by trying every c-subset of the tile
    bool cap_search = false;    // plan with several gate caps per pass, keep the plan with the fewest passes
    bool fuse_1q = true; // multiply chains of single-qubit ops on one qubit (FP64, host)
    bool staged = true;  // build register-staged programs for the tile kernel
    bool c64 = false;    // complex64 state: passes become dense 5-qubit tensor-core blocks
    int max_gates_per_pass = 96;  // keeps a pass program within the kernel parameter
    bool dense2_reg = false;  // dense two-qubit gates as register ops (SOP_U2) rather than shared-memory ops
};

struct PlannedPass {
    std::vector<int> tile;       // tile qubits (logical ids), ascending physical position
    std::vector<int> phys_in;    // physical position of tile bit t (ascending)
    std::vector<int> out_tile;   // input tile bit t is written to tile bit out_tile[t]
    std::vector<int> gates;      // indices into Plan::pgates executed by this pass
    std::vector<DevOp> ops;      // device ops, tile-relative (generic kernel)
    std::vector<int> phys_before;  // layout (logical -> physical) when the pass starts
    std::shared_ptr<PassProg> prog;  // register-staged program (tile kernel), if it applies
    std::shared_ptr<BlockProg> bprog;  // complex64 tensor-core block program, if it applies
    std::string prog_note;           // why the generic kernel runs this pass, if it does
};

// FP64 instructions per amplitude that the pass-specialised kernel spends
// on register-staged op `o` (DFMA, DMUL, DADD as generated; NOTs are
// register moves or address flips).
inline double sop_fp64_per_amp(const SOp& o) {
    switch (o.kind) {
    case SOP_U: return 8;                                       // 2 DMUL + 6 DFMA
    case SOP_UR: case SOP_UX: return 4;                         // 2 DMUL + 2 DFMA
    case SOP_URA: case SOP_URB: case SOP_UXA: case SOP_UXB: return 2;  // 2 DFMA
    case SOP_H: return 3;                                       // 2 DADD + 2 DMUL + 2 DFMA per pair
    case SOP_U2: return 16;                                     // 2 DMUL + 14 DFMA
    case SOP_D1: case SOP_DR: return 4;                         // complex multiply
    case SOP_PH: return 4.0 / (double)(1u << __builtin_popcount(o.creg));
    default: return 0;
    }
}

// A gate as the planner sees it (logical qubits).
struct PGate {
    int kind = 0;             // OPK_* from device_types.h
    std::vector<int> tq;      // target qubits, in gate-bit order
    std::vector<int> fq;      // free qubits (controls, or diagonal qubits in bit order)
    std::vector<Cx> table;    // dense matrix (row-major) or diagonal table
    double ph_re = 1.0, ph_im = 0.0;
    int src = -1;             // index in the program's gate list
};

struct Plan {
    int n = 0;
    bool dense2_reg = false;         // PlanOptions::dense2_reg of the plan
    std::vector<PGate> pgates;
    std::vector<PlannedPass> passes;
    std::vector<int> final_phys;     // logical qubit -> physical bit after the last pass
    std::vector<int> label_to_logical;  // program label x holds logical qubit label_to_logical[x] at the end
    std::vector<int> initial_permutation, final_inverse_permutation;
    std::vector<Cx> pool;            // dense matrices and diagonal tables of all ops
    std::vector<DevOp> smem_ops;     // shared-memory ops referenced by register-staged programs
    std::vector<uint8_t> bimg;       // complex64 block operand images (KATE_BLOCK_IMG_BYTES each)
};

// Classifies gates, plans passes and lowers them to device ops. Dense gates
// above 5 qubits are rejected (message returned).
std::string build_plan(const Program& prog, const PlanOptions& opt, Plan* out);

// Remap-only passes taking layout `phys` (logical -> physical) to `target`.
std::vector<PlannedPass> plan_relayout(int n, const std::vector<int>& phys, const std::vector<int>& target,
                                       const PlanOptions& opt);

// Register-staged program of a pass (12-qubit tiles). Non-register ops are
// appended to smem_ops (their tables to pool). Returns "" on success.
// low_first: the first stage takes no register among tile bits 0..3 while
// it has ops without them, so that its lanes 0..3 can read HBM in 256-byte
// runs (no copy-in through the shared tile).
std::string build_pass_program(const Plan& plan, const PlannedPass& pass, int n, std::vector<DevOp>& smem_ops,
                               std::vector<Cx>& pool, PassProg* out, bool dense2 = false, bool low_first = false);

// Shared-memory round trips of a register-staged program's tile: one per
// stage boundary, one for a copy-in when the first stage's registers hold a
// tile bit among 0..3, one for a write-back when the last stage's lanes 0..3
// are not the tile bits that go to physical bits 0..3.
int prog_round_trips(const PassProg& p);

// Complex64 block program of a pass (12-qubit tiles); operand images are
// appended to `pool`. Returns "" on success.
std::string build_block_program(const Plan& plan, const PlannedPass& pass, int n, std::vector<uint8_t>& pool,
                                BlockProg* out);
// Greedy partition of a pass's gates into blocks of at most five qubits:
// the block number of each gate.
std::vector<int> block_partition(const std::vector<PGate>& pg, const std::vector<int>& gates);

// Register-op form of a 2x2 matrix: SOP_UR (real), SOP_UX ([[a, ib], [ic, d]]) or SOP_U.
int classify_2x2(const Cx* m);

// Device descriptor of a pass whose ops start at op0.
DevPass to_devpass(int n, const PlannedPass& p, int op0);

// Lowers one pass's gates into device ops (tile-relative); matrices and
// tables are appended to `pool` (complex doubles).
void lower_pass(const Plan& plan, PlannedPass& pass, const std::vector<int>& phys, std::vector<Cx>& pool);

}  // namespace kate
