// Warp-specialised register-staged tile kernel for complex128 states (the
// plain method's group pass): the same pass programs as k_tile.cu, with the
// HBM reads decoupled from the arithmetic.
//
// One CTA per SM (persistent; each CTA takes a contiguous range of cosets):
//   producer warp (warp 8): streams the CTA's coset tiles into a ring of
//       NBUF 64 KiB shared-memory buffers with cp.async.bulk. A tile is 256
//       runs of 16 contiguous amplitudes (tile bits 0..3 are physical bits
//       0..3), one 256-byte bulk copy per run, landing in plain index order;
//       each buffer has a "full" mbarrier (transaction bytes) and an "empty"
//       one (the 8 consumer warps' arrivals);
//   consumer warps (warps 0..7, 256 threads x 16 amplitudes): wait for a
//       full buffer, run the pass program on it (register stages, exchanges
//       through the buffer), store the last stage's registers straight to
//       the state (the qubit remap applied) or, when its lanes would not
//       write 256-byte runs, through the buffer, then release the buffer.
// While the consumers compute on one tile, the next NBUF - 1 tiles are in
// flight from HBM, and the stores are fire-and-forget, so the pass runs at
// the rate of whichever is slower, HBM or the program, instead of their sum.
// At 288 threads per SM the consumers may hold up to 224 registers, so the
// interpreter's 16 amplitudes and tables stay in registers (no spills).
//
// All mbarrier waits are bounded (%globaltimer): a wait that runs out sets
// the error flag for the host (kate_sim_synchronize reports it); the
// consumers leave together (barrier with an OR vote) and the producer waits,
// again bounded, for the copies it issued before returning.
// Replaces, like k_tile.cu, the reference's per-group kernel
// (HIPcode/simulator.hpp:143-218) and its per-gate switch
// (HIPcode/GPUGate.hpp:21-203).
#include "k_stage.cuh"
#include "launch.hpp"

namespace kate {

namespace {

using namespace stage;

constexpr int NCONS = 256;               // consumer threads
constexpr int NTHR = NCONS + 32;         // + producer warp
constexpr uint32_t TILE_BYTES = TS * 16;  // 64 KiB
constexpr uint32_t RUN_BYTES = 256;       // 16 amplitudes
constexpr unsigned long long WAIT_NS = 2000000000ull;

template <int NBUF>
struct WsLayout {
    static constexpr size_t tables = (size_t)NBUF * TILE_BYTES;
    static constexpr size_t direct = tables + sizeof(TileTables<double2>);
    static constexpr size_t bars = (direct + sizeof(DirectIO) + 7) & ~(size_t)7;
    static constexpr size_t total = bars + 2 * NBUF * 8 + 16;  // full[], empty[], abort flag
};

__device__ __forceinline__ uint64_t gtime() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of parity `parity` to complete; false when the wait
// ran out or another warp raised the abort flag.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, const volatile int* abort) {
    if (mbar_try(a, parity)) return true;
    const uint64_t t0 = gtime();
    for (uint32_t it = 1;; it++) {
        if (mbar_try(a, parity)) return true;
        if ((it & 63u) == 0) {
            if (*abort) return false;
            if (gtime() - t0 > WAIT_NS) return false;
        }
    }
}
// One bulk copy global -> shared, completing `bytes` transaction bytes on
// the mbarrier at shared address mbar.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
// Consumer barrier with an OR vote over the 256 consumer threads.
__device__ __forceinline__ bool cons_bar_or(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 256, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

template <int NBUF>
__global__ void __launch_bounds__(NTHR, 1)
    k_tile_ws(double2* __restrict__ st, const __grid_constant__ PassProg P, int* __restrict__ err) {
    using L = WsLayout<NBUF>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TileTables<double2>& T = *reinterpret_cast<TileTables<double2>*>(smem_raw + L::tables);
    DirectIO& D = *reinterpret_cast<DirectIO*>(smem_raw + L::direct);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + L::bars);
    volatile int* abort = reinterpret_cast<volatile int*>(bars + 2 * NBUF);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t full0 = (uint32_t)__cvta_generic_to_shared(bars);
    const uint32_t empty0 = full0 + 8u * NBUF;
    const uint32_t t = threadIdx.x;

    if (t < NCONS) {
        const ProgView v = view(P);
        setup_program(T, v, t);
        setup_io(T, v, t);
        setup_direct(D, v, t);
    } else if (t == NCONS) {
        for (int s = 0; s < NBUF; s++) {
            mbar_init(full0 + 8u * s, 1);
            mbar_init(empty0 + 8u * s, NCONS / 32);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const uint32_t ncos = 1u << P.ncb;
    const uint32_t c_begin = (uint32_t)((uint64_t)blockIdx.x * ncos / gridDim.x);
    const uint32_t c_end = (uint32_t)((uint64_t)(blockIdx.x + 1) * ncos / gridDim.x);

    if (t >= NCONS) {
        // ---- producer warp ----
        const uint32_t lane = t - NCONS;
        // Run r = lane + 32 k holds tile bits 4..11 = r: lanes give tile bits
        // 4..8, k tile bits 9..11.
        uint64_t loff = 0;
        for (int i = 0; i < 5; i++)
            if ((lane >> i) & 1u) loff |= 1ull << P.tphys[4 + i];
        uint64_t koff[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            uint64_t o = 0;
            for (int i = 0; i < 3; i++)
                if ((k >> i) & 1) o |= 1ull << P.tphys[9 + i];
            koff[k] = o;
        }
        uint32_t issued = 0;
        bool ok = true;
        for (uint32_t c = c_begin; c < c_end; c++, issued++) {
            const uint32_t s = issued % NBUF, ph = (issued / NBUF) & 1u;
            // A fresh barrier's preceding phase (parity 1) counts as complete.
            if (lane == 0) ok = mbar_wait(empty0 + 8u * s, ph ^ 1u, abort);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            const uint32_t fb = full0 + 8u * s;
            if (lane == 0) mbar_arrive_tx(fb, TILE_BYTES);
            __syncwarp();
            const double2* src = st + (coset_base(T, c) | loff);
            const uint32_t dst = sbase + s * TILE_BYTES + lane * RUN_BYTES;
#pragma unroll
            for (int k = 0; k < 8; k++) bulk_g2s(dst + (uint32_t)k * 32u * RUN_BYTES, src + koff[k], RUN_BYTES, fb);
        }
        if (!ok && lane == 0) {
            atomicExch(err, 1);
            *abort = 1;
        }
        // Never leave with copies in flight: wait for the last load of every
        // buffer (bounded; these complete unless the memory system failed).
        if (lane == 0) {
            const uint32_t first = issued > (uint32_t)NBUF ? issued - NBUF : 0u;
            for (uint32_t i = first; i < issued; i++) {
                const uint64_t t0 = gtime();
                while (!mbar_try(full0 + 8u * (i % NBUF), (i / NBUF) & 1u))
                    if (gtime() - t0 > WAIT_NS) {
                        atomicExch(err, 1);
                        break;
                    }
            }
        }
        return;
    }

    // ---- consumer warps ----
    const int nops = P.nops;
    const bool copy_out = !D.okS;
    uint32_t i = 0;
    for (uint32_t c = c_begin; c < c_end; c++, i++) {
        const uint32_t s = i % NBUF, ph = (i / NBUF) & 1u;
        const bool ok = mbar_wait(full0 + 8u * s, ph, abort);
        if (cons_bar_or(!ok)) {
            if (t == 0) {
                atomicExch(err, 1);
                *abort = 1;
            }
            break;
        }
        const uint32_t tb = sbase + s * TILE_BYTES;
        double2* tile = reinterpret_cast<double2*>(smem_raw + (size_t)s * TILE_BYTES);
        run_program<double2, false, 5, 1>(T, nops, tb, tile, coset_base(T, c), nullptr, 0, nullptr, t, &D, st);
        if (copy_out) {
            prog_bar<1>();
            store_tile<double2, false>(T, st, c, tb, t);
        }
        // This thread's shared-memory accesses of the buffer come before the
        // next bulk copy into it (async proxy), then the warp releases it.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if ((t & 31u) == 0) mbar_arrive(empty0 + 8u * s);
    }
}

static_assert(WsLayout<3>::total <= 227 * 1024, "three tile buffers and the tables fit one SM");

// SM count of `device`, after raising the kernel's shared-memory limit there
// (once per device).
template <int NBUF>
int ws_grid_for(int device) {
    static int cached[64] = {0};
    if (device < 0 || device >= 64) device = 0;
    if (!cached[device]) {
        cudaFuncSetAttribute(k_tile_ws<NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WsLayout<NBUF>::total);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cached[device] = sms;
    }
    return cached[device];
}

}  // namespace

bool tile_ws_applies(const PassProg& prog) {
    if (prog.m != TB || prog.ncb > 22 || prog.nstages < 1) return false;
    for (int i = 0; i < 4; i++)
        if (prog.tphys[i] != i) return false;
    bool staged = false;
    for (int k = 0; k < prog.nops; k++) {
        const int kind = prog.ops[k].kind;
        if (kind == SOP_SMEM) return false;
        if (kind == SOP_STAGE) staged = true;
        else if (!staged && kind != SOP_XL && kind != SOP_XF) return false;  // register ops before any load
    }
    return staged;
}

int tile_ws_grid(int n, int device) {
    const int g = ws_grid_for<3>(device);
    const uint64_t ncos = 1ull << (n - TB);
    return (int)(ncos < (uint64_t)g ? ncos : (uint64_t)g);
}

cudaError_t launch_tile_ws(void* st, const PassProg& prog, int* err, int grid, cudaStream_t s) {
    if (!tile_ws_applies(prog)) return cudaErrorInvalidValue;
    int dev = 0;
    cudaGetDevice(&dev);
    ws_grid_for<3>(dev);
    k_tile_ws<3><<<grid, NTHR, WsLayout<3>::total, s>>>((double2*)st, prog, err);
    return cudaGetLastError();
}

}  // namespace kate
