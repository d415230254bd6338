// Pass-specialised group-pass kernels (complex128).
//
// The register-staged tile kernel (k_tile.cu) interprets a pass program: per
// op it loads the op from shared memory, switches on its kind and register
// bit, and runs one of several unrolled bodies. On B200 that costs about
// three instructions of dispatch, branching and register moves per FP64
// instruction. This generator instead turns a pass program into CUDA source
// in which every op is straight-line code on named registers: register bits,
// shared-memory and HBM offsets and loop bounds are compile-time constants;
// matrices stay data (a __grid_constant__ parameter read from the constant
// bank), so passes of the same shape share one kernel. The source is
// compiled for sm_100a with NVRTC when a simulator is created and cached per
// device by its text. The arithmetic of each op is the interpreter's, op for
// op, so both paths compute the same amplitudes.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "device_types.h"

namespace kate {

// CUDA source of the kernel for `prog`, or "" (with *why set) when the
// program has a form the generator does not take (shared-memory ops, a
// register op before the first stage). from_zero: the pass is the first of
// a run from |0...0>; it generates its input instead of loading it (only
// coset 0 is nonzero; every other coset's output is zero, written without
// being read), so the run needs no separate initialisation pass.
// occ: CTAs per SM the kernel is compiled for (launch bounds; each CTA
// holds a 64 KiB exchange tile, so at most 3).
// form 2: the first pass of a run from a product state (execute with
// per-qubit (theta, phi)): its input is computed, as amplitude = prod_p
// v[bit p][p] (coset factor times two 64-entry tile tables), from a second
// parameter (ProdTab), so no initialisation pass runs and the state is not
// read.
std::string jit_pass_source(const PassProg& prog, std::string* why, int form = 0, int occ = 2);

// Compiles the sources not yet cached on `device` (in parallel) and returns
// a kernel handle per source. Returns "" on success.
std::string jit_compile(int device, const std::vector<std::string>& srcs, std::vector<void*>* fns);

// The fields of `prog` that its generated source depends on (everything but
// the matrix values), with from_zero and occ: a key a few KB long, so a
// simulator whose passes were compiled before finds their kernels without
// generating their sources (about 0.2 ms per pass).
std::string jit_pass_key(const PassProg& prog, int form, int occ);
// The kernel compiled on `device` for a pass key, or null.
void* jit_find(int device, const std::string& key);
// Records the kernel of a pass key (from jit_compile).
void jit_remember(int device, const std::string& key, void* fn);

// Work per amplitude of the kernel jit_pass_source generates for `prog`
// (form 0): FP64 instructions (DFMA, DMUL, DADD as emitted; NOTs are
// register moves or address flips and count nothing) and shared-memory
// bytes moved (16 B stored and 16 B loaded per amplitude for each stage
// exchange, for a copy-in through the tile and for a write-back through
// it). False when the generator does not take the program.
bool jit_pass_work(const PassProg& prog, double* fp64_per_amp, double* smem_bytes_per_amp);

// Local memory (register spill) bytes per thread of a compiled kernel; -1
// when unknown.
int jit_local_bytes(void* fn);

// Grid of a pass-specialised kernel for 2^ncb cosets on `device`.
int jit_grid(int ncb, int device);

// Launches kernel fn (from jit_compile) on the complex128 state st with the
// matrices of prog.
cudaError_t jit_launch(void* fn, void* st, const PassProg& prog, int grid, cudaStream_t s);
// The per-qubit factors of a form-2 kernel: v[b][p] multiplies amplitudes
// whose physical bit p is b.
struct ProdTab {
    double2 v[2][KATE_MAX_QUBITS];
};
cudaError_t jit_launch_prod(void* fn, void* st, const PassProg& prog, const ProdTab& pt, int grid, cudaStream_t s);

}  // namespace kate
