// Serving engine: a stream of circuit requests, continuous batching on one
// GPU.
//
// The reference runs one circuit per Simulator, blocking the calling thread
// (HIPcode/simulator.hpp:301-353, execute). A Server instead owns an engine
// thread. submit() queues a request (circuit, shots, seed) and returns at
// once; host threads plan it (the same planning as a Batch); the engine
// admits planned requests in submission order while their states fit the
// HBM budget (a buddy allocator over one device arena), and then runs steps:
// each step is one launch of the batch kernel (k_batch.cu) in which every
// scheduled request advances by some of its remaining levels (group passes,
// then <Z> and chunk sums, their prefix, and inverse-CDF sampling), so
// requests join and leave between steps and small ones finish while large
// ones are still running. Results (<Z_q> and the samples, in program-label
// order like kate_sim_sample) are kept until collected.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "batch.hpp"
#include "circuit.hpp"

namespace kate {

struct ServeOptions {
    uint64_t budget_bytes = 150ull << 30;  // resident states (the admission budget)
    uint64_t aux_bytes = 2ull << 30;       // programs, outputs, sums, uniforms
    int64_t step_tiles = 1 << 16;          // tile passes per step before requests wait for the next one
    int step_latency_us = 1500;            // estimated critical path of one step (0: no limit)
    int chunk = 4;                         // cosets per pass task
    int zchunks = 4;                       // 2^16-amplitude chunks per <Z> task
    int schunks = 16;                      // chunks per sampling task
    int planners = 0;                      // planning threads (0: hardware concurrency, at most 16)
    BatchTune tune;                        // planning choices for every request
};

struct ServeResult {
    int n = 0;
    std::vector<double> z;          // <Z> per program label
    std::vector<uint64_t> samples;  // basis-state indices in label order, ascending CDF order
    std::vector<uint8_t> zbit;      // internal: physical bit of each label (samples are converted on collection)
    double t_submit = 0, t_admit = 0, t_done = 0;  // seconds since the server started
};

struct ServerImpl;

class Server {
public:
    static std::string create(int precision, int device, const ServeOptions& opt, Server** out);
    ~Server();  // stops the engine after the running step; pending requests are dropped

    // Queues a request; thread-safe; does not block on the GPU.
    std::string submit(const Program& p, int shots, uint64_t seed, int64_t* id);
    // Waits up to timeout_s for request id and moves its result out.
    // Returns "timeout" when it is not done yet.
    std::string wait(int64_t id, double timeout_s, ServeResult* out);
    // Counters: [0] submitted [1] completed [2] live [3] queued [4] steps
    // [5] resident bytes [6] peak resident bytes [7] failed; engine thread
    // time in microseconds: [8] admission [9] step building [10] step
    // launch to completion [11] result collection.
    void stats(int64_t* out) const;
    double now() const;  // seconds since the server started

private:
    ServerImpl* d_ = nullptr;
};

}  // namespace kate
