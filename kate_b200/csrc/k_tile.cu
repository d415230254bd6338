// Register-staged tile kernel: one group pass over the state, for complex128
// (FP64 arithmetic, 64 KiB tiles) and complex64 (FP32 arithmetic, 32 KiB
// tiles) amplitudes. The program machinery is in k_stage.cuh.
//
// Each CTA (256 threads) owns one 4096-amplitude coset tile at a time, in a
// grid-stride loop over cosets:
//   1. the tile is copied global -> shared with 16-byte cp.async (each warp
//      instruction reads runs of 2^c contiguous amplitudes, c >= 4); the
//      copies of the next cosets are issued before the current one is
//      processed (a ring of up to three buffers, one CTA per SM), so HBM
//      reads overlap compute;
//   2. the pass program runs: a register stage loads 16 amplitudes per
//      thread from shared memory, applies its ops in registers (2x2, H,
//      controlled X, controlled phase, one-qubit diagonal), and stores them
//      back at the next stage boundary; shared-memory ops (dense blocks,
//      multi-qubit diagonals) run between stages;
//   3. the tile is written back to global with its tile bits permuted (the
//      qubit remap), again in contiguous runs.
// The program is a __grid_constant__ kernel parameter, copied into shared
// memory by every CTA. This replaces the reference's
// per-group kernel (HIPcode/simulator.hpp:143-218) and its per-gate device
// switch (HIPcode/GPUGate.hpp:21-203).
#include "k_stage.cuh"
#include "launch.hpp"

namespace kate {

namespace {

using namespace stage;

// Complex128 with one buffer also keeps the DirectIO tables (first-stage
// loads and last-stage stores straight to global memory).
template <typename C2, int NBUF>
constexpr bool tile_direct() {
    return sizeof(C2) == 16 && NBUF == 1;
}

template <typename C2, int NBUF>
constexpr size_t tile_smem_bytes() {
    return (size_t)NBUF * TS * sizeof(C2) + sizeof(TileTables<C2>) + (tile_direct<C2, NBUF>() ? sizeof(DirectIO) : 0);
}

// SM: whether the program has shared-memory ops (the variant without them
// has no call in its loop, so nothing is spilled around it). NBUF tile
// buffers: NBUF = 1, two CTAs per SM overlap each other's load and compute
// phases; NBUF = 2 or 3, one CTA per SM keeps the next NBUF - 1 cosets'
// copies in flight while it processes the current one (one cp.async group
// per iteration, empty when there is nothing left to prefetch, so the group
// count stays uniform).
template <typename C2, bool SM, int NBUF>
__global__ void __launch_bounds__(NT, NBUF == 1 ? 2 : 1)
    k_tile(C2* __restrict__ st, const __grid_constant__ PassProg P, const DevOp* __restrict__ sops,
           const double2* __restrict__ pool) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2* bufs = reinterpret_cast<C2*>(smem_raw);
    TileTables<C2>& T = *reinterpret_cast<TileTables<C2>*>(bufs + NBUF * TS);
    DirectIO* D = tile_direct<C2, NBUF>() ? reinterpret_cast<DirectIO*>(&T + 1) : nullptr;
    const uint32_t t = threadIdx.x;
    {
        const ProgView v = view(P);
        setup_program(T, v, t);
        setup_io(T, v, t);
        if constexpr (tile_direct<C2, NBUF>()) setup_direct(*D, v, t);
    }
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(bufs);
    __syncthreads();
    const uint32_t ncos = 1u << P.ncb;
    const int nops = P.nops, sop0 = P.sop0;
    constexpr uint32_t BUF_BYTES = TS * sizeof(C2);
    // NBUF = 1: grid-stride over cosets. NBUF > 1: each CTA takes a
    // contiguous range of cosets, so the tiles it has in flight together are
    // neighbours in memory (coset bit 0 is usually physical bit c), which
    // lengthens the DRAM runs beyond 2^c amplitudes.
    const uint32_t c_begin = NBUF == 1 ? blockIdx.x : (uint32_t)((uint64_t)blockIdx.x * ncos / gridDim.x);
    const uint32_t c_end = NBUF == 1 ? ncos : (uint32_t)((uint64_t)(blockIdx.x + 1) * ncos / gridDim.x);
    const uint32_t c_step = NBUF == 1 ? gridDim.x : 1u;
    if (NBUF > 1) {
        for (int k = 0; k < NBUF - 1; k++) {
            const uint32_t c = c_begin + k;
            if (c < c_end) load_async(T, st, c, sbase + k * BUF_BYTES, t);
            else asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
    }
    // Tile copies through shared memory unless the first (last) stage reads
    // (writes) global memory itself.
    const bool copy_in = !tile_direct<C2, NBUF>() || !D->okL;
    const bool copy_out = !tile_direct<C2, NBUF>() || !D->okS;
    int it = 0;
    for (uint32_t c = c_begin; c < c_end; c += c_step, it++) {
        const int slot = NBUF == 1 ? 0 : it % NBUF;
        const uint32_t tb = sbase + (uint32_t)slot * BUF_BYTES;
        C2* tile = bufs + slot * TS;
        if (NBUF > 1) {
            // Prefetch the coset NBUF - 1 iterations ahead into the buffer the
            // previous iteration released, then wait for this one.
            const uint32_t cn = c + (NBUF - 1);
            if (cn < c_end) load_async(T, st, cn, sbase + (uint32_t)((it + NBUF - 1) % NBUF) * BUF_BYTES, t);
            else asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group %0;\n" ::"n"(NBUF - 1) : "memory");
        } else if (copy_in) {
            load_async(T, st, c, sbase, t);
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        if (copy_in) __syncthreads();
        run_program<C2, SM>(T, nops, tb, tile, coset_base(T, c), sops, sop0, pool, t, D, st);
        if (copy_out) {
            __syncthreads();
            store_tile<C2, false>(T, st, c, tb, t);
        }
        // The buffer is rewritten by the next coset (only in the same warps'
        // slots when every exchange is warp-local).
        if (tile_direct<C2, NBUF>() && D->wl) __syncwarp();
        else __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

}  // namespace

template <typename C2, int NBUF>
int tile_grid_for(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        const int smem = (int)tile_smem_bytes<C2, NBUF>();
        cudaFuncSetAttribute(k_tile<C2, true, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_tile<C2, false, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<C2, false, NBUF>, NT, smem);
        if (occ < 1) occ = 1;
        cached[device] = sms * occ;
    }
    return cached[device];
}

template <typename C2>
cudaError_t launch_tile_t(void* st, const PassProg& prog, const DevOp* sops, const void* pool, int grid, int nbuf,
                          cudaStream_t s) {
    if (prog.m != TB || prog.ncb > 22) return cudaErrorInvalidValue;
    bool sm = false;
    for (int k = 0; k < prog.nops; k++) sm |= prog.ops[k].kind == SOP_SMEM;
    C2* x = (C2*)st;
    const double2* pl = (const double2*)pool;
    if (nbuf == 3) {
        const size_t smem = tile_smem_bytes<C2, 3>();
        if (sm) k_tile<C2, true, 3><<<grid, NT, smem, s>>>(x, prog, sops, pl);
        else k_tile<C2, false, 3><<<grid, NT, smem, s>>>(x, prog, sops, pl);
    } else if (nbuf == 2) {
        const size_t smem = tile_smem_bytes<C2, 2>();
        if (sm) k_tile<C2, true, 2><<<grid, NT, smem, s>>>(x, prog, sops, pl);
        else k_tile<C2, false, 2><<<grid, NT, smem, s>>>(x, prog, sops, pl);
    } else {
        const size_t smem = tile_smem_bytes<C2, 1>();
        if (sm) k_tile<C2, true, 1><<<grid, NT, smem, s>>>(x, prog, sops, pl);
        else k_tile<C2, false, 1><<<grid, NT, smem, s>>>(x, prog, sops, pl);
    }
    return cudaGetLastError();
}

int tile_pass_grid(int n, int device, int nbuf, int prec) {
    int g;
    if (prec == 1)
        g = nbuf == 3 ? tile_grid_for<float2, 3>(device)
                      : nbuf == 2 ? tile_grid_for<float2, 2>(device) : tile_grid_for<float2, 1>(device);
    else
        g = nbuf == 3 ? tile_grid_for<double2, 3>(device)
                      : nbuf == 2 ? tile_grid_for<double2, 2>(device) : tile_grid_for<double2, 1>(device);
    const uint64_t ncos = 1ull << (n - TB);
    return (int)(ncos < (uint64_t)g ? ncos : (uint64_t)g);
}

cudaError_t launch_tile(void* st, int prec, const PassProg& prog, const DevOp* sops, const void* pool, int grid,
                        int nbuf, cudaStream_t s) {
    if (prec == 1) return launch_tile_t<float2>(st, prog, sops, pool, grid, nbuf, s);
    return launch_tile_t<double2>(st, prog, sops, pool, grid, nbuf, s);
}

}  // namespace kate
