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
};

struct BatchOptions {
    int chunk = 4;                // cosets per PASS task
    int zchunks = 4;              // 2^16-amplitude chunks per ZRED task
    uint64_t window_bytes = 0;    // queue large circuits in windows of this many state bytes (0: one window)
    std::vector<BatchTune> tune;  // by qubit count (index n); missing entries use the defaults
    const BatchTune& for_n(int n) const;
};

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

private:
    BatchImpl* d_ = nullptr;
};

// Chooses BatchTune per qubit count present in `circuits` by timing
// candidate plans of a sample of those circuits on the device.
std::string batch_autotune(const std::vector<const Program*>& circuits, int precision, int device, BatchOptions* opt);

}  // namespace kate
