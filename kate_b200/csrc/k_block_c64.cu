// Complex64 group pass with 5-qubit dense blocks on the tensor cores
// (tcgen05, kind::f16 with BF16 operands, split-BF16 products, FP32
// accumulation in TMEM); the block arithmetic is in k_block.cuh.
//
// Each CTA (256 threads; two CTAs per SM, ~97 KiB of shared memory each)
// processes 4096-amplitude coset tiles in a grid-stride loop, with two
// staging buffers: while a tile is processed, the next one is already being
// copied in (16-byte cp.async of amplitude pairs; tile bit 0 is physical
// bit 0), so the HBM load latency is hidden behind the blocks. The block
// matrices (B operands, hi and lo) are staged in shared memory once per
// CTA. All waits are bounded: on timeout the kernel records an error flag
// for the host and returns after its copies in flight completed, freeing
// its TMEM.
#include <cuda_runtime.h>

#include "k_block.cuh"
#include "launch.hpp"

namespace kate {

namespace {

using namespace blk;

constexpr uint32_t OFF_B = 0;                                                   // blocks' B images
constexpr uint32_t OFF_S = OFF_B + KATE_C64_MAX_BLOCKS * KATE_BLOCK_IMG_BYTES;  // two staging tiles
constexpr uint32_t OFF_MISC = OFF_S + 2 * S_BYTES;  // products' mbarrier, TMEM slot, abort flag, images' mbarrier
constexpr uint32_t OFF_TAB = OFF_MISC + 64;
constexpr uint32_t OFF_IO = OFF_TAB + TAB_BYTES;
constexpr uint32_t SMEM_BYTES = OFF_IO + IO_BYTES + 1024;  // + alignment slack

__global__ void __launch_bounds__(NT, 2)
    k_block_c64(float2* __restrict__ st, const __grid_constant__ BlockProg P, const uint8_t* __restrict__ bimg,
                int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-byte aligned operand region
    uint8_t* gbase = smem_raw + (base - raw);
    const uint32_t t = threadIdx.x;
    const uint32_t mbar = base + OFF_MISC;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + OFF_MISC + 8);
    int* abort_flag = reinterpret_cast<int*>(gbase + OFF_MISC + 16);
    uint16_t* tab = reinterpret_cast<uint16_t*>(gbase + OFF_TAB);
    uint16_t* iot = reinterpret_cast<uint16_t*>(gbase + OFF_IO);

    const uint32_t mbar_img = base + OFF_MISC + 24;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_img) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *abort_flag = 0;
    }
    tmem_alloc(tmem_slot, TMEM_COLS);
    __syncthreads();
    // Block matrices: B images into shared memory once, by the bulk-copy engine.
    uint32_t phase_img = 0;
    if (!load_images(P.nblocks, [&](int b) { return bimg + P.bimg[b]; }, base + OFF_B, mbar_img, phase_img) &&
        t == 0)
        *abort_flag = 1;
    Pass X;
    setup(P, tab, iot, X);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const uint64_t ncos = 1ull << P.ncb;
    uint32_t phase = 0;
    auto load = [&](uint64_t c, int buf) {
        // One cp.async group per tile (an empty one past the last coset, so
        // every iteration waits for exactly its own tile).
        if (c < ncos) load_tile<false>(st, coset_base(P, c), base + OFF_S + (uint32_t)buf * S_BYTES, X, iot);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    load(blockIdx.x, 0);
    int it = 0;
    for (uint64_t c = blockIdx.x; c < ncos; c += gridDim.x, it++) {
        const int cur = it & 1;
        float2* S = reinterpret_cast<float2*>(gbase + OFF_S + (uint32_t)cur * S_BYTES);
        // The other buffer was last read by the previous tile's write-back,
        // which the barrier at the end of that iteration closed.
        load(c + gridDim.x, cur ^ 1);
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        float2* const SS[1] = {S};
        if (!apply_blocks<1>(P, X, tab, SS, base + OFF_B, tmem, mbar, phase, abort_flag)) break;
        store_tile<false>(P, X, iot, st, coset_base(P, c), S);
        __syncthreads();
    }
    if (*abort_flag && t == 0) atomicExch(err, 1);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    tmem_free(tmem, TMEM_COLS);
}

}  // namespace

int block_c64_grid(int n, int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        cudaFuncSetAttribute(k_block_c64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        cudaFuncSetAttribute(k_block_c64, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        int sms = 148, smem_sm = 0, reserved = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
        // Registers allow two CTAs (__launch_bounds__); shared memory decides.
        int occ = smem_sm / (int)(SMEM_BYTES + reserved);
        if (occ < 1) occ = 1;
        if (occ > 2) occ = 2;
        cached[device] = sms * occ;
    }
    const uint64_t ncos = 1ull << (n - TB);
    return (int)(ncos < (uint64_t)cached[device] ? ncos : (uint64_t)cached[device]);
}

cudaError_t launch_block_c64(void* st, const BlockProg& prog, const void* bimg, int* err, int grid, cudaStream_t s) {
    if (prog.m != TB || prog.nblocks < 1 || prog.nblocks > KATE_C64_MAX_BLOCKS) return cudaErrorInvalidValue;
    if (prog.tphys[0] != 0) return cudaErrorInvalidValue;  // amplitude pairs must be contiguous
    k_block_c64<<<grid, NT, SMEM_BYTES, s>>>((float2*)st, prog, (const uint8_t*)bimg, err);
    return cudaGetLastError();
}

}  // namespace kate
