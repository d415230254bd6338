// Plain structs shared by the host planner and the CUDA kernels.
#pragma once

#include <stdint.h>

#define KATE_MAX_QUBITS 40
#define KATE_MAX_TILE 14

// Device op kinds.
#define OPK_DENSE 0  // dense 2^k x 2^k on tile bits tb[0..k-1] (bit i of local index <-> tb[i])
#define OPK_H 1      // Hadamard on tile bit tb[0], with the reference's arithmetic
#define OPK_X 2      // NOT on tile bit tb[0] where all controls are 1 (CNOT, TOFFOLI)
#define OPK_PHASE 3  // multiply by (ph_re, ph_im) where all controls are 1 (CRk)
#define OPK_DIAG 4   // multiply by table[sum_i bit_i << i], bit i from ftb[i] (tile) or fpos[i] (coset)

typedef struct {
    int32_t kind;
    int32_t k;         // dense / diag qubit count
    int32_t tb[5];     // target tile bits (dense bit order), tb[0] for H / X
    int32_t ftb[5];    // diag qubit i: tile bit, or -1 when outside the tile
    int32_t fpos[5];   // diag qubit i outside the tile: physical bit
    uint32_t tmask;    // controls inside the tile (tile-bit mask)
    uint64_t pmask;    // controls outside the tile (physical-bit mask)
    int64_t mat;       // offset into the matrix pool, in complex elements
    double ph_re, ph_im;
} DevOp;

// ---- Register-staged pass program (the tile kernel's instruction stream) ----
// A pass is a sequence of stages. A register stage holds 16 amplitudes per
// thread (256 threads x 16 = the 4096-amplitude tile): register-index bit i
// is tile bit rb[i], thread-index bit i is tile bit tb[i]. Single-qubit ops
// whose target is a register bit run on registers; controls and diagonal
// bits may be register, thread or coset bits. Anything else runs as a
// shared-memory op between register stages.
#define SOP_STAGE 1  // store registers (if a stage is open), sync (a warp barrier when src = 1), load with rb/tb
#define SOP_SMEM 2   // generic op on the shared-memory tile (DevOp index idx)
#define SOP_U 3      // 2x2 on register bit a; matrix mats[idx .. idx+3] (row-major)
#define SOP_H 4      // Hadamard on register bit a (the reference's arithmetic)
#define SOP_X 5      // NOT on register bit a where controls creg/cthr/ccos are all 1
#define SOP_PH 6     // multiply by mats[idx] where controls creg/cthr/ccos are all 1
#define SOP_D1 7     // multiply by mats[idx + bit]; bit from register/thread/coset bit a (src)
#define SOP_UR 8     // 2x2 with real entries on register bit a: mats[idx..idx+3].x (4 FP64 ops/amplitude)
#define SOP_UX 9     // 2x2 [[a, ib], [ic, d]] (a, b, c, d real) on register bit a: 4 FP64 ops/amplitude
#define SOP_DR 10    // diagonal over the register bits: multiply register j by mats[idx + j]
#define SOP_XF 11    // fold a NOT into the stage's store: store offset ^= idx where controls cthr/ccos are 1
#define SOP_XL 12    // fold a NOT into the next stage's load: load offset ^= idx where controls cthr/ccos are 1
// Rotations with a common factor taken out of the matrix (one FMA-class op
// per real component of an amplitude instead of two). mats[idx] = (t0, t1);
// the factors of a pass are multiplied together and applied once, folded
// into one diagonal or full 2x2 op of the same pass (a scalar commutes with
// every op). On register bit a, x0 / x1 the pair's amplitudes:
#define SOP_URA 13   // x0' = x0 + t0 x1,     x1' = t1 x0 + x1      (real [[a, b], [c, a]] / a)
#define SOP_URB 14   // x0' = t0 x0 + x1,     x1' = t1 x1 - x0      (real [[a, b], [-b, d]] / b)
#define SOP_UXA 15   // x0' = x0 + i t0 x1,   x1' = x1 + i t1 x0    ([[a, ib], [ic, a]] / a)
#define SOP_UXB 16   // x0' = x1 - i t0 x0,   x1' = x0 - i t1 x1    ([[a, ib], [ib, d]] / (ib))
// Dense two-qubit gate on register bits a (local index bit 0) and src (bit
// 1), a < src; matrix mats[idx .. idx+15] (4x4 complex, row-major). Only in
// complex128 plans (PlanOptions::dense2_reg).
#define SOP_U2 17

#define SRC_REG 0
#define SRC_THR 1
#define SRC_COS 2

#define KATE_TILE_BITS 12
#define KATE_MAX_SOPS 160
#define KATE_MAX_MATS 640
#define KATE_MAX_STAGES 40

typedef struct {
    uint8_t kind;
    uint8_t a;       // register bit (U/H/X; D1 SRC_REG), thread bit (D1 SRC_THR) or physical bit (D1 SRC_COS)
    uint8_t src;     // D1 source
    uint8_t creg;    // controls on register bits (register-index mask)
    uint8_t cthr;    // controls on thread bits (thread-index mask)
    uint8_t pad;
    uint16_t idx;    // mats index (U, PH, D1, DR), DevOp index (SMEM) or stage index (STAGE)
    uint64_t ccos;   // controls on coset bits (physical-bit mask)
} SOp;               // 16 bytes: one shared-memory vector load per op

typedef struct {
    int32_t m, ncb, nops, nmats;
    uint8_t tphys[16];
    uint8_t outsrc[16];
    uint8_t cphys[48];
    SOp ops[KATE_MAX_SOPS];
    double mats[KATE_MAX_MATS][2];
    // Per stage (SOP_STAGE idx): byte offsets in the swizzled tile, with
    // s0(t) = stab[idx][t & 15] ^ stab[idx][16 + (t >> 4)] the thread's
    // base and W_k(j) the XOR of stab[idx][32 + 4k + i] over the set bits i
    // of register index j:
    //   load  register j from  s0(t) ^ L(t) ^ W_0(j)   (L: SOP_XL flips)
    //   store register j to    s0(t) ^ S(t) ^ W_1(j)   (S: SOP_XF flips)
    //   natural layout          s0(t) ^ W_2(j)
    // NOTs and CNOTs on register bits at the start (end) of a stage commute
    // into an affine map of the register index that the load (store)
    // addressing applies, so they move no data.
    uint16_t stab[KATE_MAX_STAGES][44];
    // Per stage: tile bit of register-index bit i (rb) and of thread-index
    // bit i (tb), the layout the tables above encode.
    uint8_t srb[KATE_MAX_STAGES][4];
    uint8_t stb[KATE_MAX_STAGES][8];
    int32_t nstages;
    int32_t sop0;    // first shared-memory op of this pass in the simulator's array (SMEM idx is relative)
} PassProg;

typedef struct {
    int32_t m;          // tile bits
    int32_t nops;
    int32_t op0;        // first op index
    int32_t ncb;        // coset bits = n - m
    uint8_t tphys[16];  // physical bit of tile bit t (ascending)
    uint8_t outsrc[16]; // on store, output tile bit t takes input tile bit outsrc[t]
    uint8_t cphys[48];  // physical bits of the coset index, ascending
} DevPass;

// ---- complex64 tensor-core pass program (k_block_c64.cu) ----
// A pass applies up to KATE_C64_MAX_BLOCKS dense 5-qubit blocks to each
// 4096-amplitude tile. Block b acts on tile bits btb[b][0..4] (ascending;
// bit i of the block's local index is btb[b][i]); its 32x32 complex matrix
// is stored as the real 64x64 matrix W (W[2r][2c] = Re U[r][c],
// W[2r][2c+1] = -Im U[r][c], W[2r+1][2c] = Im U[r][c], W[2r+1][2c+1] =
// Re U[r][c]) split into BF16 hi and lo parts (hi = bf16(w), lo =
// bf16(w - hi)), each laid out as the K-major SWIZZLE_128B UMMA operand
// image (64 rows x 128 B: 8 KiB), hi then lo: KATE_BLOCK_IMG_BYTES per block
// at byte offset bimg[b] of the image pool.
#define KATE_C64_MAX_BLOCKS 2
#define KATE_BLOCK_IMG_BYTES 16384

// The staging tile's layout: element e (tile index) sits at position
// e ^ sum_k parity(e & smask[k]) << k (k = 0..3, masks over tile bits 4..11:
// linear over GF(2) and invertible), chosen per pass so that a warp's rows
// (a block's 4 lowest non-block tile bits) and its write-back lanes fall on
// distinct 8-byte bank pairs. smask[0] = 0 keeps amplitude pairs (e, e + 1)
// side by side in one 16-byte slot.
typedef struct {
    int32_t m, ncb, nblocks, pad;
    uint8_t tphys[16];
    uint8_t outsrc[16];
    uint8_t cphys[48];
    uint8_t btb[KATE_C64_MAX_BLOCKS][8];
    uint64_t bimg[KATE_C64_MAX_BLOCKS];
    uint16_t smask[4];
} BlockProg;

// ---- batched execution (k_batch.cu) ----
// A batch is a task list run by one persistent kernel. SMALL tasks simulate
// a whole circuit of at most KATE_BATCH_SMALL_MAX qubits (narrower circuits
// are padded with idle qubits) in one CTA's shared memory: |0...0>, every
// pass program back to back on the same tile, then <Z_q>. PASS tasks run one
// group pass over a range of cosets of a larger circuit's state; ZRED tasks
// add a range of a finished state's amplitudes into its <Z_q> outputs. Tasks
// are queued level by level (pass index) per circuit, and a task waits until
// `need` tasks of its circuit have finished, so it only ever waits on tasks
// taken from the queue before it.
#define KATE_BATCH_SMALL_MAX 12
#define KATE_BATCH_MAX_QUBITS 28
#define BT_SMALL 0
#define BT_PASS 1
#define BT_ZRED 2    // also writes per-chunk probability sums when the circuit has psum storage
#define BT_PREFIX 3  // exclusive prefix of the chunk sums (one task per circuit)
#define BT_SAMPLE 4  // inverse-CDF sampling of the shots that fall in a range of chunks

typedef struct {
    int32_t kind;
    int32_t circ;
    int32_t prog;     // BT_PASS: program index; BT_SMALL: first program index
    int32_t nprog;    // BT_SMALL: programs run back to back
    uint32_t c0, c1;  // BT_PASS: coset range; BT_ZRED / BT_SAMPLE: range of 2^16-amplitude chunks
    int32_t need;     // finished tasks of this circuit required before starting
    int32_t first;    // BT_PASS: the input is |0...0> (nothing is loaded)
} BatchTask;

typedef struct {
    uint64_t off;     // state offset in the arena (amplitudes)
    int32_t n;        // qubits: <Z> outputs, and 2^n amplitudes for the reductions
    int32_t shots;    // samples to draw (BT_SAMPLE)
    int64_t zoff;     // first <Z> output of this circuit
    int64_t poff;     // chunk sums at psum[poff + ch], their exclusive prefix at psum[poff + nch + ch],
                      // the total at psum[poff + 2 nch]; -1: no sums
    int64_t uoff;     // the shots' uniforms in [0, 1), ascending: unif[uoff + s]
    int64_t soff;     // sampled (physical) amplitude indices: sout[soff + s]
    uint8_t zbit[40]; // output q reads bit zbit[q] of the tile (SMALL) or state (otherwise)
} BatchCirc;

// A pass program in the batch's program blob: a register-staged program
// (nstages >= 0: SOp ops, double[2] matrices, stage tables) or, when none
// could be built, a generic one (nstages < 0: DevOp ops run on the shared
// tile one by one). Offsets are in bytes from the blob's start.
#define BPROG_SMEM 1  // BatchProg.flags: the staged program has SOP_SMEM ops
// BatchProg.flags: a complex64 tensor-core block pass. ops_off is the blob
// offset of its BlockProg, whose bimg[b] are block b's operand images as
// byte offsets from that BlockProg (so the pair moves as one).
#define BPROG_BLOCK 2

typedef struct {
    int32_t m, ncb, nops, nmats, nstages, sop0;  // sop0: first shared-memory op in the batch's array
    int32_t flags, pad;
    uint8_t tphys[16];
    uint8_t outsrc[16];
    uint8_t cphys[48];
    uint64_t ops_off, mats_off, stab_off;
} BatchProg;
