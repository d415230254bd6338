// Host-side launchers of the CUDA kernels (defined in the .cu files).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "device_types.h"

namespace kate {

// Product-state initialisation value table: v[b][p] is the factor for
// physical bit p having value b.
struct ProductInit {
    double v[2][KATE_MAX_QUBITS][2];
    int n;
};

// prec: 0 = complex128 (double2 amplitudes), 1 = complex64 (float2).
cudaError_t launch_set_basis0(void* st, uint64_t dim, int prec, cudaStream_t s);
cudaError_t launch_init_product(void* st, int n, const ProductInit& P, int prec, cudaStream_t s);
cudaError_t launch_pass_generic(void* st, int prec, const DevPass& p, const DevOp* ops, const void* pool, int grid,
                                cudaStream_t s);
cudaError_t launch_bitsums(const void* st, int prec, int n, int kind, void* partials, cudaStream_t s);
cudaError_t launch_probs(const void* st, int prec, uint64_t dim, double* out, cudaStream_t s);
// Renormalisation of a complex64 state (n >= 1 qubits): ||psi||^2 reduced in
// FP64 on the device, then every amplitude multiplied by 1 / ||psi||. The
// scratch (renorm_scratch_bytes(), zeroed once) holds the per-CTA partials,
// then ||psi||^2 and 1 / ||psi|| as doubles 0 and 1 after the partials
// (offset renorm_result_offset()), then a counter.
size_t renorm_scratch_bytes();
// Inverse-CDF sampling on the device (k_sample.cu): unif holds `shots`
// uniforms in [0, 1), ascending; out[s] receives the physical index of the
// first amplitude whose FP64 cumulative probability exceeds unif[s] * total.
// scratch: sample_scratch_doubles(n) doubles.
size_t sample_scratch_doubles(int n);
cudaError_t launch_sample(const void* st, int prec, int n, const double* unif, int shots, double* scratch,
                          uint64_t* out, cudaStream_t s);
// Device gate merger (k_merge.cu): out[b] is the product of blocks[b] as one
// dense gate on the sorted union of its qubits (at most 10), bit-identical
// to merge_gates (circuit.hpp); all blocks in one launch on `device`, then
// a synchronise of `stream`. Returns "" or an error message.
struct Gate;
std::string merge_gates_device(const std::vector<std::vector<Gate>>& blocks, int device, cudaStream_t stream,
                               std::vector<Gate>* out);
constexpr size_t renorm_result_offset() { return 148 * 4 * sizeof(double); }
cudaError_t launch_renorm_c64(void* st, int n, void* scratch, cudaStream_t s);

// c128 state (double2 amplitudes)
cudaError_t launch_set_basis0_c128(void* st, uint64_t dim, cudaStream_t s);
cudaError_t launch_init_product_c128(void* st, int n, const ProductInit& P, cudaStream_t s);
// One generic group pass (shared-memory tile, any op mix). Dense ops up to 5 qubits.
cudaError_t launch_pass_generic_c128(void* st, int n, const DevPass& p, const DevOp* ops, const void* pool,
                                     int grid, cudaStream_t s);
int generic_pass_grid(int n, int m, int device);
// Register-staged tile kernel (12-qubit tiles, 256 threads x 16 amplitudes),
// prec 0: complex128 / FP64, 1: complex64 / FP32. nbuf = 2: one CTA per SM
// with a prefetched second tile; nbuf = 1: two CTAs per SM with one tile each.
cudaError_t launch_tile(void* st, int prec, const PassProg& prog, const DevOp* sops, const void* pool, int grid,
                        int nbuf, cudaStream_t s);
int tile_pass_grid(int n, int device, int nbuf, int prec);
// Warp-specialised complex128 tile kernel (k_tile_ws.cu): one CTA per SM, a
// producer warp streaming tiles with bulk copies into a ring of shared-memory
// buffers. Applies to register-staged programs without shared-memory ops
// whose tile holds physical bits 0..3. err: device int set to 1 if a bounded
// wait gave up.
bool tile_ws_applies(const PassProg& prog);
int tile_ws_grid(int n, int device);
cudaError_t launch_tile_ws(void* st, const PassProg& prog, int* err, int grid, cudaStream_t s);

// Complex64 pass of 5-qubit dense blocks on the tensor cores. err: device
// int set to 1 if a bounded wait gave up.
cudaError_t launch_block_c64(void* st, const BlockProg& prog, const void* bimg, int* err, int grid, cudaStream_t s);
int block_c64_grid(int n, int device);

// Persistent batch kernel (k_batch.cu). head, done[circuits], zout (large
// circuits' outputs) must be zero at launch; err is set to 1 when a
// dependency wait gave up after wait_ns (the kernel then stops). psum /
// unif / sout: chunk sums, uniforms and samples of circuits that sample (may
// be null otherwise).
cudaError_t launch_batch(void* arena, int prec, const BatchTask* tasks, int ntasks, const BatchCirc* circs,
                         const BatchProg* progs, const void* blob, const DevOp* sops, const void* pool, int* head,
                         int* done, double* zout, int* err, int grid, cudaStream_t s, double* psum = nullptr,
                         const double* unif = nullptr, uint64_t* sout = nullptr,
                         unsigned long long wait_ns = 5000000000ull, int tensor_blocks = 0);
int batch_grid(int device, int prec, bool tensor_blocks = false);

// Bit sums: per CTA, for every local bit, the sum over amplitudes with the
// bit 0 and with the bit 1, plus the total. kind 0 sums amplitudes (double2
// partials), kind 1 sums |a|^2 (double partials). Returns the grid shape.
struct BitSumShape {
    int grid;   // CTAs (2^g)
    int g;      // coset bits handled by the grid
    int nr;     // round bits handled per thread
    int nout;   // partial values per CTA
};
BitSumShape bitsum_shape(int n);
cudaError_t launch_bitsums_c128(const void* st, int n, int kind, void* partials, cudaStream_t s);
// Amplitude bit sums with an explicit shape: 2^g CTAs, nr round bits per
// thread (n = 12 + g + nr when n >= 12), partials of 1 + 2 * (12 + nr)
// double2 per CTA.
cudaError_t launch_bitsums_c128_shape(const void* st, int n, int g, int nr, void* partials, cudaStream_t s);
cudaError_t launch_probs_c128(const void* st, uint64_t dim, double* out, cudaStream_t s);

}  // namespace kate
