// Persistent batch kernel: many independent circuits in one launch.
//
// CTAs take tasks from a global queue (one atomicAdd per task). A task
// first waits, with a time-bounded spin, until the tasks of its circuit that
// it depends on have finished (per-circuit counters), then runs:
//   BT_SMALL  the whole circuit in shared memory: |0...0>, every pass
//             program back to back on the same tile, <Z_q>; the state never
//             touches HBM;
//   BT_PASS   one group pass program over a range of cosets: 16-byte
//             cp.async loads (L2 only: other SMs wrote the state earlier in
//             this launch), the register-staged program, stores that bypass
//             L1. The first pass of a circuit starts from |0...0> in shared
//             memory instead of loading;
//   BT_ZRED   <Z_q> partial sums over a range of amplitudes, added to the
//             circuit's outputs with FP64 atomics (and, for sampling, each
//             chunk's probability sum);
//   BT_PREFIX exclusive prefix of a circuit's chunk sums;
//   BT_SAMPLE inverse-CDF sampling of the shots falling in a chunk range.
// Finished tasks bump their circuit's counter after a memory fence. Tasks
// are queued level by level per circuit, so a task waits only on tasks
// dequeued before it: every CTA that holds a task can finish it, whatever
// the number of resident CTAs.
// C2 is the amplitude type: float2 (complex64, FP32 arithmetic) or double2
// (complex128, FP64 arithmetic). <Z> sums are FP64.
#include <cuda_runtime.h>

#include "k_block.cuh"
#include "k_stage.cuh"
#include "launch.hpp"

namespace kate {

namespace {

using namespace stage;


__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    return v;
}

__device__ __forceinline__ double2 ldst(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldst(const float2* p) {
    const float2 v = __ldcg(p);
    return make_double2(v.x, v.y);
}

// Block-wide sums of per-thread values v[0..nb): result in red[NB * 8 + b].
template <int NB>
__device__ void block_sums(const double (&v)[NB], int nb, double* red) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        if (b >= nb) break;
        double x = v[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp * NB + b] = x;
    }
    __syncthreads();
    if (t < nb) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; w++) s += red[w * NB + t];
        red[NB * (NT / 32) + t] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ ProgView view(const BatchProg& P, const unsigned char* blob) {
    ProgView v;
    v.m = P.m;
    v.ncb = P.ncb;
    v.nops = P.nstages >= 0 ? P.nops : 0;  // generic programs run from global memory
    v.nmats = P.nstages >= 0 ? P.nmats : 0;
    v.nstages = P.nstages >= 0 ? P.nstages : 0;
    v.sop0 = P.sop0;
    v.tphys = P.tphys;
    v.outsrc = P.outsrc;
    v.cphys = P.cphys;
    v.ops = reinterpret_cast<const SOp*>(blob + P.ops_off);
    v.mats = reinterpret_cast<const double(*)[2]>(blob + P.mats_off);
    v.stab = reinterpret_cast<const uint16_t(*)[44]>(blob + P.stab_off);
    return v;
}

// Dynamic shared memory of the batch kernel: two tiles, then the program
// tables or, for a tensor-core block task, the block region: the B operand
// images (1024-byte aligned), the BlockProg, the block tables.
extern __shared__ __align__(16) unsigned char batch_smem_raw[];
constexpr uint32_t BLK_IMG = KATE_C64_MAX_BLOCKS * KATE_BLOCK_IMG_BYTES;
constexpr uint32_t BLK_PROG = (sizeof(BlockProg) + 15) & ~15u;
constexpr uint32_t BLK_REGION = 1024 + BLK_IMG + BLK_PROG + blk::TAB_BYTES + blk::IO_BYTES;
static_assert(sizeof(BlockProg) % 8 == 0, "BlockProg is copied as 8-byte words");
// Per CTA, for the whole launch (complex64 batches with block programs):
// the products' mbarrier and its phase, the TMEM columns, the wait flag.
__shared__ uint64_t blk_mbar, blk_mbar_img;
__shared__ uint32_t blk_tmem, blk_phase, blk_phase_img;
__shared__ int blk_abort;

// A complex64 tensor-core block pass over cosets [c0, c1) of one circuit
// (the BatchProg's BPROG_BLOCK program): the BlockProg and its operand
// images into shared memory, then per coset the staging tile (loaded, or
// the tile of |0...0> for a circuit's first pass), the blocks, the
// write-back. The two batch tile buffers are the double-buffered staging
// tiles. Loads and stores go through L2 only (other SMs wrote the state
// earlier in this launch). Returns false when a product wait gave up.
__device__ __noinline__ bool block_task(float2* st, const BatchProg& BP, const unsigned char* blob, uint32_t c0,
                                        uint32_t c1, bool first) {
    const uint32_t t = threadIdx.x;
    const uint32_t tmem = blk_tmem, mbar = blk::smem_u32(&blk_mbar);
    int* abort_flag = &blk_abort;
    uint32_t phase = blk_phase;  // every thread keeps the same copy; thread 0 stores it back
    unsigned char* raw = batch_smem_raw + 2 * TS * sizeof(float2);
    const uint32_t rawa = blk::smem_u32(raw);
    const uint32_t bbase = (rawa + 1023u) & ~1023u;
    unsigned char* g = raw + (bbase - rawa);
    BlockProg& P = *reinterpret_cast<BlockProg*>(g + BLK_IMG);
    uint16_t* tab = reinterpret_cast<uint16_t*>(g + BLK_IMG + BLK_PROG);
    uint16_t* iot = reinterpret_cast<uint16_t*>(g + BLK_IMG + BLK_PROG + blk::TAB_BYTES);
    const unsigned char* src = blob + BP.ops_off;
    for (uint32_t i = t; i < sizeof(BlockProg) / 8; i += NT)
        reinterpret_cast<uint64_t*>(&P)[i] = __ldcg(reinterpret_cast<const unsigned long long*>(src) + i);
    __syncthreads();
    // The operand images by the bulk-copy engine (the previous task's
    // products, the last readers of this region, completed before it ended).
    uint32_t phase_img = blk_phase_img;
    const bool img_ok = blk::load_images(P.nblocks, [&](int b) { return src + P.bimg[b]; }, bbase,
                                         blk::smem_u32(&blk_mbar_img), phase_img);
    if (!img_ok) *abort_flag = 1;
    blk::Pass X;
    blk::setup(P, tab, iot, X);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float2* S0 = reinterpret_cast<float2*>(batch_smem_raw);
    const uint32_t sb0 = blk::smem_u32(batch_smem_raw);
    bool ok = true;
    if (first) {
        for (uint32_t c = c0; c < c1 && ok; c++) {
            const uint64_t cb = blk::coset_base(P, c);
            blk::zero_tile(S0, cb == 0);
            __syncthreads();
            float2* const SS[1] = {S0};
            ok = blk::apply_blocks<1>(P, X, tab, SS, bbase, tmem, mbar, phase, abort_flag);
            if (ok) blk::store_tile<true>(P, X, iot, st, cb, S0);
            __syncthreads();
        }
        if (t == 0) {
            blk_phase = phase;
            blk_phase_img = phase_img;
        }
        return ok;
    }
    blk::load_tile<true>(st, blk::coset_base(P, c0), sb0, X, iot);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    uint32_t it = 0;
    for (uint32_t c = c0; c < c1; c++, it++) {
        const uint32_t cur = it & 1u;
        float2* S = S0 + cur * TS;
        // The other buffer was last read by the previous tile's write-back,
        // closed by the barrier at the end of that iteration.
        if (c + 1 < c1) blk::load_tile<true>(st, blk::coset_base(P, c + 1), sb0 + (cur ^ 1u) * blk::S_BYTES, X, iot);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        float2* const SS[1] = {S};
        if (!blk::apply_blocks<1>(P, X, tab, SS, bbase, tmem, mbar, phase, abort_flag)) {
            ok = false;
            break;
        }
        blk::store_tile<true>(P, X, iot, st, blk::coset_base(P, c), S);
        __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
        blk_phase = phase;
        blk_phase_img = phase_img;
    }
    return ok;
}

// The register-staged program as a call of its own, so that its registers
// are allocated apart from the task loop's. The tile and tables are taken
// from the shared-memory symbol (shared-window addressing).
template <typename C2, bool SM>
__device__ __noinline__ void run_staged(int nops, uint64_t cbase, const DevOp* __restrict__ sops, int sop0,
                                        const double2* __restrict__ pool, uint32_t boff) {
    C2* tile = reinterpret_cast<C2*>(batch_smem_raw + boff);
    const TileTables<C2>& T = *reinterpret_cast<const TileTables<C2>*>(batch_smem_raw + 2 * TS * sizeof(C2));
    const uint32_t tb = (uint32_t)__cvta_generic_to_shared(tile);
    run_program<C2, SM>(T, nops, tb, tile, cbase, sops, sop0, pool, threadIdx.x);
}

// Runs program P (tables already in T) on the tile, for coset base cbase.
template <typename C2>
__device__ __forceinline__ void run_any(const TileTables<C2>& T, const BatchProg& P, const unsigned char* blob,
                                        uint32_t tb, C2* tile, uint64_t cbase, const DevOp* __restrict__ sops,
                                        const double2* __restrict__ pool, uint32_t t) {
    if (P.nstages >= 0) {
        const uint32_t boff = tb - (uint32_t)__cvta_generic_to_shared(batch_smem_raw);
        if (P.flags & BPROG_SMEM) run_staged<C2, true>(P.nops, cbase, sops, P.sop0, pool, boff);
        else run_staged<C2, false>(P.nops, cbase, sops, P.sop0, pool, boff);
    } else {
        const DevOp* gops = reinterpret_cast<const DevOp*>(blob + P.ops_off);
        for (int k = 0; k < P.nops; k++) {
            const DevOp op = gops[k];
            ops::apply_op<C2>(tile, TB, cbase, op, pool, (int)t, NT);
            __syncthreads();
        }
    }
}

// <Z_q> of a resident tile: output q reads tile bit zbit[q].
template <typename C2>
__device__ __noinline__ void small_z(const C2* tile, int nz, const uint8_t* zbit, double* red, double* out) {
    const uint32_t t = threadIdx.x;
    double z[KATE_BATCH_SMALL_MAX];
#pragma unroll
    for (int q = 0; q < KATE_BATCH_SMALL_MAX; q++) z[q] = 0.0;
    for (uint32_t i = t; i < (uint32_t)TS; i += NT) {
        const C2 a = tile[ops::tsw<C2>(i)];
        const double p = (double)a.x * a.x + (double)a.y * a.y;
#pragma unroll
        for (int q = 0; q < KATE_BATCH_SMALL_MAX; q++)
            if (q < nz) z[q] += ((i >> zbit[q]) & 1u) ? -p : p;
    }
    block_sums<KATE_BATCH_SMALL_MAX>(z, nz, red);
    if ((int)t < nz) out[t] = red[KATE_BATCH_SMALL_MAX * (NT / 32) + t];
}

// <Z_q> partial sums of an n-qubit state over 2^16-amplitude chunks
// [ch0, ch1), added to out[q] (q reads physical bit zbit[q]). Thread t takes
// amplitudes chunk * 2^16 + t + 256 k: physical bits 0..7 come from t, 8..15
// from k, the rest from the chunk. With psum, also stores each chunk's
// probability sum at psum[ch] (block-reduced in a fixed order).
template <typename C2>
__device__ __noinline__ void zred(const C2* st, int n, uint32_t ch0, uint32_t ch1, const uint8_t* zbit, double* red,
                                  double* out, double* psum) {
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    double z[KATE_BATCH_MAX_QUBITS];
#pragma unroll
    for (int q = 0; q < KATE_BATCH_MAX_QUBITS; q++) z[q] = 0.0;
    for (uint32_t ch = ch0; ch < ch1; ch++) {
        double tot = 0.0, kb[8];
#pragma unroll
        for (int b = 0; b < 8; b++) kb[b] = 0.0;
        const uint64_t x0 = (uint64_t)ch << 16;
        for (uint32_t k = 0; k < 256; k++) {
            const uint64_t x = x0 + t + ((uint64_t)k << 8);
            if (x >> n) break;
            const double2 a = ldst(st + x);
            const double p = a.x * a.x + a.y * a.y;
            tot += p;
#pragma unroll
            for (int b = 0; b < 8; b++) kb[b] += ((k >> b) & 1u) ? -p : p;
        }
#pragma unroll
        for (int b = 0; b < KATE_BATCH_MAX_QUBITS; b++) {
            if (b < 8) z[b] += ((t >> b) & 1u) ? -tot : tot;
            else if (b < 16) z[b] += kb[b - 8];
            else z[b] += ((ch >> (b - 16)) & 1u) ? -tot : tot;
        }
        if (psum) {
            double w = tot;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
            if (lane == 0) red[warp] = w;
            __syncthreads();
            if (t == 0) {
                double sc = 0.0;
                for (int i = 0; i < NT / 32; i++) sc += red[i];
                psum[ch] = sc;
            }
            __syncthreads();
        }
    }
    block_sums<KATE_BATCH_MAX_QUBITS>(z, n, red);
    if ((int)t < n) atomicAdd(out + t, red[KATE_BATCH_MAX_QUBITS * (NT / 32) + zbit[t]]);
}

// Block-wide exclusive scan of one double per thread (fixed order); also
// returns the block total.
__device__ double block_exscan(double v, double* red, double* total) {
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    double x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) red[warp] = x;
    __syncthreads();
    if (t == 0) {
        double s = 0.0;
        for (int i = 0; i < NT / 32; i++) {
            const double w = red[i];
            red[i] = s;
            s += w;
        }
        red[NT / 32] = s;
    }
    __syncthreads();
    const double r = red[warp] + x - v;
    *total = red[NT / 32];
    __syncthreads();
    return r;
}

// Exclusive prefix of nch chunk sums psum[0..nch) into psum[nch..2 nch),
// the total into psum[2 nch].
__device__ __noinline__ void chunk_prefix(double* psum, uint32_t nch, double* red) {
    const uint32_t t = threadIdx.x;
    const uint32_t per = (nch + NT - 1) / NT, b0 = t * per, b1 = min(nch, b0 + per);
    double loc = 0.0;
    for (uint32_t c = b0; c < b1; c++) loc += psum[c];
    double total;
    double run = block_exscan(loc, red, &total);
    for (uint32_t c = b0; c < b1; c++) {
        psum[nch + c] = run;
        run += psum[c];
    }
    if (t == 0) psum[2 * nch] = total;
}

// Inverse-CDF sampling over chunks [ch0, ch1): shot s (uniforms u ascending)
// targets x = u * total; it falls in chunk ch when pre[ch] <= x < pre[ch] +
// sum[ch] (targets at or past the total go to the last chunk). Inside a
// chunk, thread t owns a contiguous run of amplitudes; a block scan of the
// runs' sums locates each target's run, whose owner walks it.
template <typename C2>
__device__ __noinline__ void sample_chunks(const C2* st, int n, uint32_t ch0, uint32_t ch1, const double* psum,
                                           const double* unif, int shots, uint64_t* out, double* red, int* srange) {
    const uint32_t t = threadIdx.x;
    const uint64_t dim = 1ull << n;
    const uint32_t nch = (uint32_t)(dim >> 16 ? dim >> 16 : 1);
    const double total = psum[2 * nch];
    for (uint32_t ch = ch0; ch < ch1; ch++) {
        const double lo_v = psum[nch + ch];
        const double hi_v = lo_v + psum[ch];
        const bool last = ch + 1 == nch;
        if (t == 0) {
            int lo = 0, hi = shots;  // first s with u_s * total >= lo_v
            while (lo < hi) {
                const int m = (lo + hi) >> 1;
                if (unif[m] * total >= lo_v) hi = m;
                else lo = m + 1;
            }
            int e = lo, e1 = shots;  // first s with u_s * total >= hi_v
            if (!last)
                while (e < e1) {
                    const int m = (e + e1) >> 1;
                    if (unif[m] * total >= hi_v) e1 = m;
                    else e = m + 1;
                }
            srange[0] = lo;
            srange[1] = last ? shots : e;
        }
        __syncthreads();
        const int s0 = srange[0], s1 = srange[1];
        __syncthreads();
        if (s0 >= s1) continue;
        const uint64_t x0 = (uint64_t)ch << 16;
        const uint64_t len = dim - x0 < (1ull << 16) ? dim - x0 : (1ull << 16);
        const uint64_t per = (len + NT - 1) / NT;
        const uint64_t a0 = x0 + (t * per < len ? t * per : len), a1 = x0 + ((t + 1) * per < len ? (t + 1) * per : len);
        double w = 0.0;
        for (uint64_t x = a0; x < a1; x++) {
            const double2 a = ldst(st + x);
            w += a.x * a.x + a.y * a.y;
        }
        double btot;
        const double base = block_exscan(w, red, &btot);
        const bool tail = (t == NT - 1) || (a1 == x0 + len);
        for (int s = s0; s < s1; s++) {
            const double y = unif[s] * total - lo_v;
            const bool mine = (y >= base && y < base + w) || (tail && y >= base + w && a1 > a0 && a1 == x0 + len);
            if (!mine || a1 <= a0) continue;
            double acc = base;
            uint64_t pick = a1 - 1;
            for (uint64_t x = a0; x < a1; x++) {
                const double2 a = ldst(st + x);
                const double p = a.x * a.x + a.y * a.y;
                acc += p;
                if (acc > y && p > 0.0) {
                    pick = x;
                    break;
                }
            }
            out[s] = pick;
        }
        __syncthreads();
    }
}

template <typename C2>
__device__ __forceinline__ void init_basis0(C2* tile, bool one, uint32_t t) {
#pragma unroll 4
    for (uint32_t i = t; i < (uint32_t)TS; i += NT) tile[i] = Amp<C2>::mk(0, 0);
    if (one && t == 0) tile[0] = Amp<C2>::mk(1, 0);  // element 0 sits at offset 0
}

// complex64: two CTAs per SM (128 registers); complex128 programs need more.
// TB (complex64 only): the batch has tensor-core block programs; the kernel
// then holds TMEM and the block region of shared memory. Batches without
// them use the kernel compiled without that code (less shared memory, more
// L1, no spills from it in the task loop).
template <typename C2, bool TB>
__global__ void __launch_bounds__(NT, sizeof(C2) == 8 ? 2 : 1)
    k_batch(C2* __restrict__ arena, const BatchTask* __restrict__ tasks, int ntasks, const BatchCirc* __restrict__ circs,
            const BatchProg* __restrict__ progs, const unsigned char* __restrict__ blob, const DevOp* __restrict__ sops,
            const double2* __restrict__ pool, int* __restrict__ head, int* __restrict__ done,
            double* __restrict__ zout, int* __restrict__ err, double* __restrict__ psum,
            const double* __restrict__ unif, uint64_t* __restrict__ sout, unsigned long long wait_ns) {
    static_assert(!TB || sizeof(C2) == 8, "tensor-core block tasks are complex64");
    // Two tile buffers (a pass task prefetches its next coset into the
    // other one), then the program tables.
    C2* tile = reinterpret_cast<C2*>(batch_smem_raw);
    TileTables<C2>& T = *reinterpret_cast<TileTables<C2>*>(batch_smem_raw + 2 * TS * sizeof(C2));
    __shared__ int s_task;
    __shared__ int s_abort;
    __shared__ uint8_t s_zbit[40];
    __shared__ int s_range[2];
    __shared__ double red[KATE_BATCH_MAX_QUBITS * (NT / 32) + KATE_BATCH_MAX_QUBITS];
    const uint32_t t = threadIdx.x;
    const uint32_t tb = (uint32_t)__cvta_generic_to_shared(tile);
    // Tensor-core block tasks (complex64 only): the CTA's TMEM columns and
    // the products' mbarrier, for the whole launch.
    if constexpr (TB) {
        {
            if (t == 0) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(blk::smem_u32(&blk_mbar)) : "memory");
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(blk::smem_u32(&blk_mbar_img)) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
                blk_abort = 0;
                blk_phase = 0;
                blk_phase_img = 0;
            }
            blk::tmem_alloc(&blk_tmem, blk::TMEM_COLS);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
    }
    for (;;) {
        if (t == 0) {
            // After a failed wait anywhere, every CTA stops at its next task.
            s_task = *((volatile int*)err) ? ntasks : atomicAdd(head, 1);
            s_abort = 0;
        }
        __syncthreads();
        const int ti = s_task;
        if (ti >= ntasks) break;
        const BatchTask K = tasks[ti];
        if (t == 0 && K.need > 0) {
            const unsigned long long t0 = now_ns();
            while (*((volatile int*)(done + K.circ)) < K.need) {
                if (now_ns() - t0 > wait_ns || *((volatile int*)err)) {
                    s_abort = 1;
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(256);
            }
            __threadfence();
        }
        if (t < 40) s_zbit[t] = circs[K.circ].zbit[t];
        __syncthreads();
        if (s_abort) break;
        const int nz = circs[K.circ].n;
        const int64_t zoff = circs[K.circ].zoff;

        bool block_pass = false;
        if constexpr (TB) block_pass = K.kind == BT_PASS && (progs[K.prog].flags & BPROG_BLOCK);
        if (block_pass) {
            if constexpr (TB) {
                if (!block_task(arena + circs[K.circ].off, progs[K.prog], blob, K.c0, K.c1, K.first != 0)) {
                    if (t == 0) atomicExch(err, 1);
                    break;
                }
            }
        } else if (K.kind == BT_SMALL || K.kind == BT_PASS) {
            // SMALL: step s runs program prog + s on the resident tile.
            // PASS: step s runs program prog on coset c0 + s.
            const bool small = K.kind == BT_SMALL;
            const int nsteps = small ? K.nprog : (int)(K.c1 - K.c0);
            C2* st = arena + circs[K.circ].off;
            if (small) {
                init_basis0(tile, true, t);
            } else {
                const ProgView v = view(progs[K.prog], blob);
                setup_program(T, v, t);
                setup_io(T, v, t);
            }
            const bool pre = !small && !K.first;  // pass task that loads: double-buffered
            if (pre) {
                __syncthreads();
                load_async(T, st, K.c0, tb, t);
            }
            for (int s = 0; s < nsteps; s++) {
                const BatchProg& P = progs[small ? K.prog + s : K.prog];
                const uint32_t c = K.c0 + (uint32_t)s;
                const uint32_t cur = pre ? (uint32_t)(s & 1) : 0u;
                const uint32_t tbc = tb + cur * (uint32_t)(TS * sizeof(C2));
                C2* tilec = tile + cur * TS;
                uint64_t cbase = 0;
                __syncthreads();
                if (small) {
                    setup_program(T, view(P, blob), t);
                } else {
                    cbase = coset_base(T, c);
                    if (K.first) {
                        init_basis0(tilec, cbase == 0, t);
                    } else if (s + 1 < nsteps) {
                        load_async(T, st, c + 1, tb + (cur ^ 1u) * (uint32_t)(TS * sizeof(C2)), t);
                        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                    } else {
                        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                    }
                }
                __syncthreads();
                run_any(T, P, blob, tbc, tilec, cbase, sops, pool, t);
                if (!small) {
                    __syncthreads();
                    store_tile<C2, true>(T, st, c, tbc, t);
                }
            }
            __syncthreads();
            if (small) small_z(tile, nz, s_zbit, red, zout + zoff);
        } else {
            const BatchCirc& C = circs[K.circ];
            const uint32_t nch = (uint32_t)(((1ull << nz) >> 16) ? ((1ull << nz) >> 16) : 1);
            if (K.kind == BT_ZRED)
                zred(arena + C.off, nz, K.c0, K.c1, s_zbit, red, zout + zoff, C.poff >= 0 ? psum + C.poff : nullptr);
            else if (K.kind == BT_PREFIX)
                chunk_prefix(psum + C.poff, nch, red);
            else if (K.kind == BT_SAMPLE)
                sample_chunks(arena + C.off, nz, K.c0, K.c1, psum + C.poff, unif + C.uoff, C.shots, sout + C.soff,
                              red, s_range);
        }
        __syncthreads();
        if (t == 0) {
            __threadfence();
            atomicAdd(done + K.circ, 1);
        }
    }
    if constexpr (TB) blk::tmem_free(blk_tmem, blk::TMEM_COLS);
}

template <typename C2, bool TB>
constexpr size_t batch_smem() {
    // Two tiles, then the tables or (TB) the tensor-core block region,
    // whichever is larger.
    return (size_t)2 * TS * sizeof(C2) +
           (TB && BLK_REGION > sizeof(TileTables<C2>) ? BLK_REGION : sizeof(TileTables<C2>));
}

}  // namespace

int batch_grid(int device, int prec, bool tensor_blocks) {
    static int cached[64][3] = {{0}};
    if (device < 0 || device >= 64) device = 0;
    const int pi = prec == 1 ? (tensor_blocks ? 2 : 1) : 0;
    if (!cached[device][pi]) {
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (pi == 2) {
            // About 100 KiB of shared memory per CTA: two CTAs per SM need
            // the largest carveout. The occupancy calculator reports one CTA
            // per SM for this kernel (it holds tcgen05 code), although two fit
            // and run together (measured: 570 against 932 ms per launch of
            // the batching workload with tensor-core block tasks).
            // __launch_bounds__ gives the registers for two; shared memory
            // decides.
            cudaFuncSetAttribute(k_batch<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batch_smem<float2, true>());
            cudaFuncSetAttribute(k_batch<float2, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
            cudaFuncAttributes fa{};
            cudaFuncGetAttributes(&fa, k_batch<float2, true>);
            int smem_sm = 0, reserved = 0;
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
            cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
            occ = smem_sm / (int)(batch_smem<float2, true>() + fa.sharedSizeBytes + reserved);
            if (occ > 2) occ = 2;
        } else if (pi == 1) {
            cudaFuncSetAttribute(k_batch<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batch_smem<float2, false>());
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<float2, false>, NT, batch_smem<float2, false>());
        } else {
            cudaFuncSetAttribute(k_batch<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batch_smem<double2, false>());
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch<double2, false>, NT,
                                                          batch_smem<double2, false>());
        }
        if (occ < 1) occ = 1;
        cached[device][pi] = sms * occ;
    }
    return cached[device][pi];
}

cudaError_t launch_batch(void* arena, int prec, const BatchTask* tasks, int ntasks, const BatchCirc* circs,
                         const BatchProg* progs, const void* blob, const DevOp* sops, const void* pool, int* head,
                         int* done, double* zout, int* err, int grid, cudaStream_t s, double* psum,
                         const double* unif, uint64_t* sout, unsigned long long wait_ns, int tensor_blocks) {
    const unsigned char* b = (const unsigned char*)blob;
    const double2* pl = (const double2*)pool;
    if (prec == 1 && tensor_blocks)
        k_batch<float2, true><<<grid, NT, batch_smem<float2, true>(), s>>>(
            (float2*)arena, tasks, ntasks, circs, progs, b, sops, pl, head, done, zout, err, psum, unif, sout, wait_ns);
    else if (prec == 1)
        k_batch<float2, false><<<grid, NT, batch_smem<float2, false>(), s>>>(
            (float2*)arena, tasks, ntasks, circs, progs, b, sops, pl, head, done, zout, err, psum, unif, sout, wait_ns);
    else
        k_batch<double2, false><<<grid, NT, batch_smem<double2, false>(), s>>>(
            (double2*)arena, tasks, ntasks, circs, progs, b, sops, pl, head, done, zout, err, psum, unif, sout, wait_ns);
    return cudaGetLastError();
}

}  // namespace kate
