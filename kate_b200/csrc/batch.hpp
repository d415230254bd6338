// Batched execution of many independent circuits in one persistent launch.
//
// The reference simulates one circuit per Simulator (CPUcode/simulator.hpp:
// 120-200, HIPcode/simulator.hpp:220-811); a caller with many small circuits
// loops over them, paying a plan, an allocation and several launches each.
// A Batch plans every circuit once (host threads), lays all states out in
// one device arena and runs the whole set as one task queue in one
// persistent kernel (k_batch.cu), captured in a CUDA graph together with the
// resets of its counters, so a run is one graph launch. Outputs are <Z_q>
// for every qubit of every circuit.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "device_types.h"

namespace kate {

// Planning choices for circuits of one qubit count.
struct BatchTune {
    int fusion = 1;      // gateFusion width for circuits without compiled instructions (1: no gateFusion)
    int max_gates = 96;  // gates per pass program
    int group = 12;      // m: qubits one pass's gates may span (gateGrouping(m)); the 12-qubit tile is filled up
    int coalesce = 4;    // c: low physical bits every pass keeps in its tile (runs of 2^c amplitudes per access)
    int blocks = 0;      // 1: complex64 states kept in HBM run their passes as 5-qubit tensor-core blocks
};

struct BatchOptions {
    int chunk = 16;               // cosets per PASS task (at most 1/16 of a circuit's cosets)
    int zchunks = 4;              // 2^16-amplitude chunks per ZRED task
    uint64_t window_bytes = 0;    // queue large circuits in windows of this many state bytes (0: one window)
    std::vector<BatchTune> tune;  // by qubit count (index n); missing entries use the defaults
    int wait_ms = 5000;           // a dependency wait in the kernel gives up after this long
    int64_t fault_task = -1;      // test hook: this task waits for a count its circuit never reaches
    const BatchTune& for_n(int n) const;
};

// One circuit, planned and packed for the batch kernel. Offsets (blob
// bytes, smem-op and pool indices) are local to the circuit.
struct CircPack {
    std::string err;
    int n_out = 0;   // the circuit's qubits: one <Z> output each
    int n_sim = 0;   // qubits simulated (narrow circuits are padded to a full tile)
    bool small = false;  // runs whole in one CTA's shared memory (BT_SMALL)
    std::vector<uint8_t> zbit;     // output x reads this bit of the final layout
    std::vector<BatchProg> progs;  // one per pass
    std::vector<uint8_t> blob;
    std::vector<DevOp> sops;
    std::vector<Cx> pool;
    std::vector<std::pair<uint64_t, int>> generic;  // (blob offset, count) of DevOp arrays
    bool blocks = false;  // its passes are tensor-core block passes (BPROG_BLOCK)
};

// Plans one circuit. resident: keep the state in device memory even when it
// would fit a tile (at least 12 qubits), so it can be sampled afterwards.
// c64: the state is complex64, so tune.blocks may turn its passes into
// tensor-core block passes (a state kept in HBM, at least 12 qubits).
std::string pack_circuit(const Program& in, const BatchTune& tune, bool resident, CircPack& out, bool c64 = false);

struct BatchImpl;

class Batch {
public:
    static std::string create(const std::vector<const Program*>& circuits, int precision, int device,
                              const BatchOptions& opt, Batch** out);
    ~Batch();

    std::string run_async(void* stream);  // one graph launch (stream: the caller's, or null for the batch's own)
    std::string synchronize();            // waits; reports a dependency wait that gave up
    std::string expect_z(double* out);    // outputs of every circuit, in circuit order (synchronizes)
    std::string time_runs(int runs, float* ms_avg);  // graph launches timed with events on the batch's stream

    int64_t num_outputs() const;
    int64_t num_tasks() const;
    uint64_t arena_bytes() const;
    int grid() const;
    int64_t num_programs() const;
    int64_t num_block_programs() const;  // pass programs run as tensor-core block passes
    // Host wall time of create() in ms: planning, assembly of the task queue,
    // device buffers and uploads, graph capture and instantiation.
    void create_times(double* ms4) const;
    uint64_t upload_bytes() const;  // host-to-device bytes copied by create()
    // Per circuit: pass programs and qubits simulated (0 for circuits run in shared memory).
    void circuit_info(int i, int* programs, int* resident_qubits) const;
    // Final state of circuit i (one with a resident state) after the last
    // run, as 2^n complex128 amplitudes in its qubit labels (synchronizes).
    std::string get_state(int i, double* out);

private:
    BatchImpl* d_ = nullptr;
};

// Chooses BatchTune per qubit count present in `circuits` by timing
// candidate plans of a sample of those circuits on the device.
std::string batch_autotune(const std::vector<const Program*>& circuits, int precision, int device, BatchOptions* opt);

}  // namespace kate
