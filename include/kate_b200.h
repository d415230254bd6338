/*
 * kate_b200.h - C ABI of the B200 state-vector gate-application path.
 *
 * Drop-in for the hot path of the Kate simulator (Line-fr/Kate): circuit
 * building, the compile passes (scheduling, fusion, grouping, allocation),
 * gate merging, simulation and measurement. The reference is a header-only
 * C++ class API with no C ABI; each entry point below names the reference
 * interface it replaces (paths within the reference project). The C++ facade
 * include/kate_b200/Kate.hpp wraps these calls with the reference's own class
 * and method names.
 *
 * Conventions (identical to the reference):
 *  - qubit q is bit q of the amplitude index (little-endian);
 *  - gate ids: 0 dense, 2 Hadamard, 3 CNOT (qbits[0] target, qbits[1]
 *    control), 4 CRk (phase e^{2 pi i / 2^k} on |11>, k = optarg),
 *    5 TOFFOLI (qbits[0], qbits[1] controls, qbits[2] target), 6 RX and
 *    7 RZ (accepted, and applied as no-ops: the reference implements no
 *    arithmetic for them; pass rotations as dense gates);
 *  - a dense gate on k qubits is a row-major 2^k x 2^k complex matrix, given
 *    as 2*4^k doubles (re, im interleaved); bit i of its local index is
 *    qbits[i];
 *  - states are 2^n complex amplitudes, (re, im) interleaved.
 *
 * Errors: every call returns a kate_status; kate_last_error() gives the
 * message of the last failure on the calling thread. The reference prints
 * and continues instead (HIPcode/HIPpreprocessor.hpp:35-40,
 * backendagnosticcode/basic_host_types.hpp:203-244).
 *
 * Ownership: host buffers are the caller's; device memory belongs to the
 * library and is released by the matching destroy call. A simulator copies
 * the program at creation, as the reference's Simulator copies its circuit
 * (HIPcode/simulator.hpp:243-270). Calls on one object are not re-entrant;
 * distinct objects may be used from distinct threads.
 */
#ifndef KATE_B200_H
#define KATE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KATE_API __attribute__((visibility("default")))
#else
#define KATE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    KATE_OK = 0,
    KATE_EINVAL = 1,   /* bad argument: qubit out of range, duplicate qubit, size mismatch */
    KATE_ENOMEM = 2,   /* device or host allocation failed, or admission budget exceeded */
    KATE_ECUDA = 3,    /* a CUDA runtime call failed (no device, launch failure, ...) */
    KATE_ETIMEDOUT = 4,/* a bounded device wait gave up */
    KATE_ESTATE = 5    /* call out of order (e.g. measuring before executing) */
} kate_status;

typedef enum {
    KATE_C128 = 0, /* complex128 state, FP64 arithmetic (the reference's only form) */
    KATE_C64 = 1   /* complex64 state; fused dense blocks on tensor cores (split-BF16 products, FP32 accumulation) */
} kate_precision;

/* Gate identifiers, as the reference defines them (backendagnosticcode/agnosticpreprocessor.hpp:28-33). */
#define KATE_DENSE 0
#define KATE_HADAMARD 2
#define KATE_CNOT 3
#define KATE_CRK 4
#define KATE_TOFFOLI 5
#define KATE_RX 6
#define KATE_RZ 7

typedef struct kate_circuit kate_circuit;
typedef struct kate_sim kate_sim;
typedef struct kate_plan kate_plan;
typedef struct kate_batch kate_batch;
typedef struct kate_server kate_server;

/* Message of the last failed call on this thread ("" if none). */
KATE_API const char* kate_last_error(void);
/* Library version string. */
KATE_API const char* kate_version(void);

/* printGpuInfo()  HIPcode/DeviceInfo.hpp:10-35: the number of CUDA devices
 * (0 when none answers), and one device's name (NUL-terminated, at most
 * name_cap bytes), global memory, shared memory per block and SM count.
 * Every output pointer is nullable. */
KATE_API kate_status kate_device_count(int* out);
KATE_API kate_status kate_device_properties(int device, char* name, int name_cap, size_t* global_mem,
                                            size_t* shared_mem_per_block, int* sm_count);

/* ---- circuit building: backendagnosticcode/QuantumCircuit.hpp:18-37 ---- */

/* Circuit(int nqbits)  QuantumCircuit.hpp:18-20. 1 <= nqbits <= 40. */
KATE_API kate_status kate_circuit_create(int nqbits, kate_circuit** out);
KATE_API kate_status kate_circuit_destroy(kate_circuit* c);
/* Deep copy (the reference passes circuits by value). */
KATE_API kate_status kate_circuit_clone(const kate_circuit* c, kate_circuit** out);
KATE_API kate_status kate_circuit_nqbits(const kate_circuit* c, int* out);

/* appendGate(Gate(id, qbits, optarg))  QuantumCircuit.hpp:25-37 with
 * basic_host_types.hpp:198-228. id must be 2..7; qubit count must match the
 * id (H 1, CNOT 2, CRk 2, TOFFOLI 3; RX/RZ 1). */
KATE_API kate_status kate_circuit_append_gate(kate_circuit* c, int id, const int* qbits, int nq, int optarg);
/* appendGate(Gate(Matrix<Complex>, qbits))  basic_host_types.hpp:229-245.
 * mat: 2*4^nq doubles, row-major, interleaved. 1 <= nq <= 10. */
KATE_API kate_status kate_circuit_append_dense(kate_circuit* c, const double* mat, const int* qbits, int nq);

/* Appends `count` gates at once (a loop of Circuit::appendGate,
 * backendagnosticcode/Circuit.hpp:71-91): gate i has id ids[i], nqs[i]
 * qubits taken in order from `qbits`, optarg optargs[i] (nullable: 0);
 * dense gates take their 4^nq complex entries (re, im) in order from
 * `dense`. All or nothing: on an error no gate is appended. */
KATE_API kate_status kate_circuit_append_many(kate_circuit* c, int count, const int* ids, const int* nqs,
                                              const int* qbits, const int* optargs, const double* dense);
KATE_API kate_status kate_circuit_num_gates(const kate_circuit* c, int* out);
/* Reads gate i. qbits receives *nq ints (capacity 64); dense (nullable)
 * receives 2*4^nq doubles for a dense gate. */
KATE_API kate_status kate_circuit_get_gate(const kate_circuit* c, int i, int* id, int* qbits, int* nq, int* optarg,
                                  double* dense);

/* ---- compile passes: backendagnosticcode/Circuit.hpp ---- */

/* gateScheduling()  Circuit.hpp:12-98 */
KATE_API kate_status kate_circuit_schedule(kate_circuit* c);
/* gateFusion(qbitsizelimit = 5, merge_time_matters = 1e-6)  Circuit.hpp:99-175 */
KATE_API kate_status kate_circuit_fuse(kate_circuit* c, int qbitsizelimit, double merge_time_matters);
/* gateGrouping(qbitgroupsize = 8)  Circuit.hpp:176-206 */
KATE_API kate_status kate_circuit_group(kate_circuit* c, int qbitgroupsize);
/* allocate(numberofgpulog2 = 0, maxlocalqbitnumber = 300)  Circuit.hpp:207-348 */
KATE_API kate_status kate_circuit_allocate(kate_circuit* c, int numberofgpulog2, int maxlocalqbitnumber);
/* compileDefault(numberofgpulog2 = 0, maxlocalqbitnumber = 300)  QuantumCircuit.hpp:126-204 */
KATE_API kate_status kate_circuit_compile_default(kate_circuit* c, int numberofgpulog2, int maxlocalqbitnumber);
/* compileOPT(5, 1e-6, 10, 0, 300)  Circuit.hpp:349-354 */
KATE_API kate_status kate_circuit_compile_opt(kate_circuit* c, int qbit_matrix_merge_size_limit, double merge_time_matters,
                                     int groupsize, int numberofgpulog2, int maxlocalqbitnumber);

KATE_API kate_status kate_circuit_num_groups(const kate_circuit* c, int* out);
/* Group i: *end = index one past its last gate, qbits (capacity 64) its
 * sorted qubit set  (QuantumCircuit.hpp:14). */
KATE_API kate_status kate_circuit_get_group(const kate_circuit* c, int i, int* end, int* qbits, int* nq);
KATE_API kate_status kate_circuit_num_instructions(const kate_circuit* c, int* out);
/* Instruction i: *kind 0 = swap pairs (qbits holds 2*pairs ints, capacity
 * 256), 1 = compute next group  (QuantumCircuit.hpp:17). */
KATE_API kate_status kate_circuit_get_instruction(const kate_circuit* c, int i, int* kind, int* qbits, int* nq);
/* initial_permutation / final_inverse_permutation, nqbits ints each;
 * *valid = 0 before compilation  (QuantumCircuit.hpp:15-16). */
KATE_API kate_status kate_circuit_get_permutations(const kate_circuit* c, int* initial, int* final_inverse, int* valid);

/* mergeGate / CPUmergeGate(gates [begin, end))  CPUcode/GateMerger.hpp:8-55,
 * HIPcode/GateMerger.hpp:43-109: the product of the gates as one dense
 * gate on the sorted union of their qubits, in FP64. out_qbits receives *k
 * ints (k <= 10), out_mat 2*4^k doubles. */
KATE_API kate_status kate_merge_gates(const kate_circuit* c, int begin, int end, int* out_qbits, int* k, double* out_mat);

/* mergeGate(to_merge, stream) on the GPU  HIPcode/GateMerger.hpp:12-109:
 * the same product as kate_merge_gates, computed on CUDA device `device`
 * on `stream` (a cudaStream_t; NULL: the default stream), one CTA per basis
 * column, and bit-identical to kate_merge_gates (every product and sum
 * rounded on its own, in the host merger's order). Returns after the
 * result is in out_mat. KATE_EINVAL without such a device: there is no
 * silent host fallback (kate_merge_gates is the host merger). */
KATE_API kate_status kate_merge_gates_device(const kate_circuit* c, int begin, int end, int device, void* stream,
                                             int* out_qbits, int* k, double* out_mat);
/* gateFusion(qbitsizelimit, merge_time_matters) with its merges on the GPU
 * (Circuit.hpp:99-175 with the merge of :168 replaced by the device merger,
 * every merged block of the pass in one launch on `device`): the same
 * intervals and bit-identical matrices as kate_circuit_fuse. */
KATE_API kate_status kate_circuit_fuse_device(kate_circuit* c, int qbitsizelimit, double merge_time_matters, int device);

/* exportqcx(filename)  Circuit.hpp:763-774 */
KATE_API kate_status kate_circuit_export_qcx(const kate_circuit* c, const char* path);

/* ---- simulation: HIPcode/simulator.hpp:220-811 ---- */

/* Simulator(circuit, 1)  HIPcode/simulator.hpp:243-300. Copies the circuit
 * (compiling it with compileDefault(0) first if it has no instructions, as
 * the reference does), plans the B200 group passes and allocates the state
 * on `device`. precision: kate_precision. */
KATE_API kate_status kate_sim_create(const kate_circuit* c, int precision, int device, kate_sim** out);
KATE_API kate_status kate_sim_destroy(kate_sim* s);

/* execute(displaytime)  HIPcode/simulator.hpp:301-353: initialise |0..0>,
 * run every instruction, measure. theta_phi (nullable) receives 2*n
 * doubles, (theta, phi) per qubit, the reference's proba_state. Blocks until
 * done. */
KATE_API kate_status kate_sim_execute(kate_sim* s, double* theta_phi);
/* execute(proba_state& in, displaytime)  HIPcode/simulator.hpp:354-406: the
 * initial state is the product state given by 2*n doubles (theta, phi). */
KATE_API kate_status kate_sim_execute_from(kate_sim* s, const double* theta_phi_in, double* theta_phi_out);

/* execute(displaytime = true)  HIPcode/simulator.hpp:301-353: the same run
 * as kate_sim_execute (theta_phi_in nullable: |0..0>; else the product state
 * of kate_sim_execute_from), with the phases the reference prints timed:
 * ms[0] initialisation and ms[1] the group passes (CUDA events on the
 * simulator's stream), ms[2] the measurement (host clock, copy included),
 * ms[3] the number of group passes. ms and theta_phi_out nullable. */
KATE_API kate_status kate_sim_execute_timed(kate_sim* s, const double* theta_phi_in, double* theta_phi_out,
                                            double* ms);

/* Asynchronous form for callers that own a CUDA stream (cudaStream_t passed
 * as void*; NULL = the simulator's own stream): initialise and run every
 * group pass, no measurement, no host synchronisation. */
KATE_API kate_status kate_sim_run_async(kate_sim* s, void* stream);
/* Waits for work queued on the simulator's streams. */
KATE_API kate_status kate_sim_synchronize(kate_sim* s);
/* Measurement of the current state (proba_state, 2*n doubles). */
KATE_API kate_status kate_sim_proba_state(kate_sim* s, double* theta_phi);

/* The full state after execution, in the reference's amplitude order
 * (its Simulator/CPUSimulator state array): 2*2^n doubles (c128), or 2*2^n
 * floats for a c64 simulator when `out` is float* (pass KATE_C64 layout).
 * For a c64 simulator the values are widened to double. */
KATE_API kate_status kate_sim_get_state(kate_sim* s, double* out);
/* Replaces the state (2*2^n doubles) - e.g. to resume from a dump. */
KATE_API kate_status kate_sim_set_state(kate_sim* s, const double* in);

/* Per-qubit <Z_q> = sum |a|^2 (1 - 2 bit_q), n doubles, FP64 reduction. */
KATE_API kate_status kate_sim_expect_z(kate_sim* s, double* out);
/* Probability of each computational basis state: 2^n doubles (n <= 30). */
KATE_API kate_status kate_sim_probabilities(kate_sim* s, double* out);
/* `shots` samples of the computational basis from |a|^2, seeded; out
 * receives shots uint64 basis indices in the reference's qubit labels.
 * Sampled on the device (any qubit count): shot k draws u_k = (the k-th
 * splitmix64 output of `seed` >> 11) * 2^-53 and takes the first index whose
 * FP64 cumulative probability exceeds u_k times the total (indices of
 * probability 0 are never drawn); only the uniforms and the samples cross
 * PCIe. The reference has no sampling; its measurement is
 * HIPcode/simulator.hpp:483-543. */
KATE_API kate_status kate_sim_sample(kate_sim* s, int shots, uint64_t seed, uint64_t* out);

/* Runs init + every pass once on the simulator's stream with a CUDA event
 * between launches and returns each pass's device time: ms[i] for pass i
 * (capacity kate_sim_num_passes), *init_ms for the initialisation. */
KATE_API kate_status kate_sim_profile_passes(kate_sim* s, float* ms, float* init_ms);
/* Number of kernels one kate_sim_run_async launches. */
KATE_API kate_status kate_sim_launches_per_run(kate_sim* s, int* out);

/* Device pointer of the state and its layout: phys[q] receives the bit
 * position currently holding qubit q (n ints). */
KATE_API kate_status kate_sim_state_device(kate_sim* s, void** dptr, int* phys);
KATE_API kate_status kate_sim_nqbits(kate_sim* s, int* out);

/* Plan introspection: number of group passes, and pass i's tile qubits
 * (capacity 16) and the number of gates it applies. */
KATE_API kate_status kate_sim_num_passes(kate_sim* s, int* out);
KATE_API kate_status kate_sim_get_pass(kate_sim* s, int i, int* tile_qbits, int* m, int* ngates);
/* Kernel that runs pass i of the simulator: 0 generic shared-memory
 * kernel, 1 register-staged interpreter, 2 pass-specialised kernel
 * (complex128; see kate_plan_pass_source), 3 complex64 tensor-core blocks.
 * Replaces the choice executeCommand makes per group instruction
 * (HIPcode/simulator.hpp:760-810). */
KATE_API kate_status kate_sim_pass_kernel(kate_sim* s, int i, int* kind);
/* Work per amplitude of pass i when its pass-specialised kernel (kind 2)
 * runs it: out3 = {HBM bytes read and written, FP64 instructions (DFMA,
 * DMUL, DADD as generated), shared-memory bytes stored and loaded}; with
 * 2^n amplitudes and the GPU's rates they bound the pass's time.
 * KATE_EINVAL for passes on other kernels. No counterpart in the
 * reference. */
KATE_API kate_status kate_sim_pass_work(kate_sim* s, int i, double* out3);
/* Complex64 simulators renormalise the state at the end of every run:
 * ||psi||^2 is reduced in FP64 on the device and every amplitude multiplied
 * by 1 / ||psi|| (the tensor-core blocks' split-BF16 products do not keep
 * the norm exactly). This returns the last run's ||psi||^2 before the
 * rescale (how far the run drifted). KATE_ESTATE before the first run,
 * KATE_EINVAL for complex128 simulators, which are not rescaled. No
 * counterpart in the reference (it has no complex64 path; its measurement,
 * HIPcode/simulator.hpp:483-543, is the FP64 reduction modelled here). */
KATE_API kate_status kate_sim_norm2_before_renorm(kate_sim* s, double* norm2);

/* ---- group-pass plans (host only, no device needed) ----
 * The single-GPU replacement for gateGrouping + allocate + the per-group
 * launches (backendagnosticcode/Circuit.hpp:176-348,
 * HIPcode/simulator.hpp:760-810): which qubits each HBM pass keeps on chip,
 * which ops it applies, and how it permutes the tile on write. */
#define KATE_PLAN_NO_REMAP 1u   /* keep the low physical bits fixed */
#define KATE_PLAN_NO_FUSE1Q 2u  /* do not multiply single-qubit chains */
#define KATE_PLAN_C64 4u        /* complex64 plan: dense 5-qubit tensor-core blocks */
#define KATE_PLAN_NO_DENSE2 8u  /* dense two-qubit gates as shared-memory ops, not register ops */
#define KATE_PLAN_REMAP_SEARCH 16u /* choose the qubits moved into the low bits by trying every subset
                                      of the tile, and the gate cap per pass among 96..144 (fewest
                                      passes): what complex128 simulators do */
KATE_API kate_status kate_plan_create(const kate_circuit* c, int max_tile, int coalesce, unsigned flags,
                                      kate_plan** out);
KATE_API kate_status kate_plan_destroy(kate_plan* p);
KATE_API kate_status kate_plan_num_passes(const kate_plan* p, int* out);
/* info[4] = {m, nops, op0, ncb}; tphys[16] physical bit of tile bit t;
 * outsrc[16]: on store, output tile bit t takes input tile bit outsrc[t]. */
KATE_API kate_status kate_plan_get_pass(const kate_plan* p, int i, int* info, uint8_t* tphys, uint8_t* outsrc);
KATE_API kate_status kate_plan_num_ops(const kate_plan* p, int* out);
/* ints[18] = {kind, k, tb[5], ftb[5], fpos[5], tmask}; *pmask; vals[2 + 2*1024]
 * = phase (re, im) then the op's matrix or diagonal table (re, im pairs).
 * kinds: 0 dense, 1 H, 2 controlled X, 3 controlled phase, 4 diagonal. */
KATE_API kate_status kate_plan_get_op(const kate_plan* p, int i, int* ints, uint64_t* pmask, double* vals);
/* Register-staged program of pass i (the PassProg struct of
 * kate_b200/csrc/device_types.h, *size bytes, copied when cap allows);
 * *has = 0 when the pass runs on the generic shared-memory kernel. */
KATE_API kate_status kate_plan_get_program(const kate_plan* p, int i, void* out, size_t cap, size_t* size, int* has);
KATE_API kate_status kate_plan_num_smem_ops(const kate_plan* p, int* out);
/* CUDA source of the pass-specialised kernel of pass i: its register-staged
 * program as straight-line code, compiled for sm_100a with NVRTC when a
 * complex128 simulator is created. from_zero 1: the form for the first
 * pass of a run from |0...0>, which generates its input; 2: the form for
 * the first pass of a run from a product state (execute(proba_state&)),
 * which computes its input from per-qubit factors (a second kernel
 * parameter). *size = bytes with
 * the terminating 0, copied when cap allows; KATE_EINVAL when the pass has
 * no such kernel (the simulator then interprets its program). Replaces the
 * reference's per-group kernel launch (HIPcode/simulator.hpp:143-218). */
KATE_API kate_status kate_plan_pass_source(const kate_plan* p, int i, int from_zero, char* out, size_t cap,
                                           size_t* size);
/* Complex64 tensor-core block program of pass i (the BlockProg struct of
 * kate_b200/csrc/device_types.h) and the pool of block operand images. */
KATE_API kate_status kate_plan_get_block_program(const kate_plan* p, int i, void* out, size_t cap, size_t* size,
                                                 int* has);
KATE_API kate_status kate_plan_block_images(const kate_plan* p, void* out, size_t cap, size_t* size);
/* Shared-memory op i of the register-staged programs, same format as kate_plan_get_op. */
KATE_API kate_status kate_plan_get_smem_op(const kate_plan* p, int i, int* ints, uint64_t* pmask, double* vals);
/* phys[q]: physical bit of logical qubit q after the last pass;
 * label_to_logical[x]: logical qubit held by program label x. */
KATE_API kate_status kate_plan_final_layout(const kate_plan* p, int* phys, int* label_to_logical);

/* ---- measurement without allocation ----
 * No counterpart in the reference: Kate allocates device memory on every
 * measurement (HIPcode/simulator.hpp:483-543 calls hipMalloc/hipFree).
 *
 * For callers that must not allocate device memory once running: a serving
 * loop that reserved the GPU's memory for resident state vectors, a caller
 * bound to a fixed budget or a memory pool it does not own, a host-language
 * binding that cannot manage device buffer lifetimes. Computes the
 * reference's per-qubit (theta, phi) of a state vector the caller already
 * holds on the current device: d_state is 2^nqbits complex128 amplitudes in
 * a device buffer of state_bytes bytes (at least 16 * 2^nqbits; a complex64
 * or shorter buffer returns KATE_EINVAL, as do a host pointer, another
 * device's pointer, a pointer not 16-byte aligned, and a state that does not
 * fit the allocation the pointer lies in); phys_of_label[x] (nullable:
 * identity) is the bit of the amplitude index holding program label x
 * (kate_sim_state_device reports it); final_inverse_permutation (nullable:
 * identity) maps labels to output qubits as in kate_sim_proba_state; both
 * must be permutations of 0..nqbits-1. theta_phi receives 2*nqbits doubles.
 * Queued on `stream` (cudaStream_t as void*, NULL = default stream) and
 * waited for before returning.
 *
 * It calls no cudaMalloc/cudaFree and no allocating library routine: its
 * scratch is one fixed __device__ array of KATE_NOALLOC_SCRATCH_BYTES bytes
 * that every GPU where the library's device code is loaded holds until the
 * process exits, so nqbits is limited to KATE_NOALLOC_MAX_QUBITS (larger
 * sizes return KATE_EINVAL). With CUDA's lazy module loading (the default)
 * the device code, and this array, is loaded on a device by the first
 * kernel launch or symbol lookup there, which can itself need device
 * memory: a caller that reserves all of a device's memory makes its first
 * call there (or runs any simulator there) before reserving it. Every call
 * looks up the array's device address (cudaGetSymbolAddress; no allocation
 * once loaded); make the first call on a device before any stream capture.
 * The array is shared by all calls and keeps the last call's contents (each
 * call writes every slot it reads); calls that overlap on the GPU race on
 * it, so the caller must serialise them. */
#define KATE_NOALLOC_MAX_QUBITS 30
#define KATE_NOALLOC_SCRATCH_BYTES 672704
KATE_API kate_status kate_proba_state_noalloc(const void* d_state, size_t state_bytes, int nqbits,
                                              const int* phys_of_label, const int* final_inverse_permutation,
                                              double* theta_phi, void* stream);

/* ---- device memory held for reuse ----
 * No counterpart in the reference, which allocates the state in every
 * Simulator constructor and frees it in the destructor
 * (HIPcode/simulator.hpp:243-300, 407-425). Here a destroyed simulator's
 * state (and a destroyed batch's arena), if at least 64 MiB, stays allocated
 * and is reused by the next simulator or batch on that device that it covers
 * (up to 4x its size), which saves the cudaMalloc / cudaFree of the whole
 * state in a loop of Simulator(circuit).execute(). At most one such buffer
 * is held per device; kate_server_create frees it before taking its budget.
 * This call frees it (device -1: on every device), e.g. before handing the
 * memory to another library. */
KATE_API kate_status kate_release_cached_memory(int device);

/* ---- batches of independent circuits ----
 * Replaces a caller's loop of `Simulator(circuit).execute()` over many
 * independent circuits (CPUcode/simulator.hpp:120-200 per circuit; the GPU
 * Simulator, HIPcode/simulator.hpp:220-811, plans, allocates and launches
 * per circuit). A batch plans every circuit once, keeps all states in one
 * device arena and runs them as one task queue in one persistent kernel,
 * captured with its counter resets in one CUDA graph: a run is one graph
 * launch. Output: <Z_q> for every qubit q of every circuit, in circuit
 * order (circuit i's outputs follow those of circuits 0..i-1), indexed like
 * kate_sim_expect_z (by program label). Circuits have 1 to
 * KATE_BATCH_MAX_QUBITS qubits; those of at most 12 run entirely in one
 * CTA's shared memory. */
#define KATE_BATCH_MAX_QUBITS 28
typedef struct {
    int fusion;    /* gateFusion width applied to circuits without groups or instructions (1: none; 0: default) */
    int max_gates; /* gates per pass program (0: default) */
    int group_qubits; /* m: qubits one pass's gates may span, 6..12, as gateGrouping(m) (0: 12) */
    int coalesce;  /* c: low physical bits every pass keeps in its tile, 1..6 (0: 4) */
    int blocks;    /* 1: complex64 circuits whose state is kept in device memory (more than 12 qubits) run
                      their passes as dense 5-qubit blocks on the tensor cores (the simulator's complex64
                      form) instead of register-staged programs; 0: register-staged */
} kate_batch_tuning;
typedef struct {
    int chunk;                 /* cosets (4096-amplitude tiles) per pass task; 0: default */
    int zchunks;               /* 65536-amplitude chunks per <Z> task; 0: default */
    unsigned long long window_bytes; /* queue large circuits in windows of this many state bytes; 0: one window */
    kate_batch_tuning tune[KATE_BATCH_MAX_QUBITS + 1]; /* by qubit count */
    int wait_ms;               /* a dependency wait in the kernel gives up after this long; 0: 5000 */
    long long fault_task;      /* test hook, 1-based: that task waits for a count never reached, so the
                                  bounded wait runs out and kate_batch_synchronize reports it; 0: none */
} kate_batch_options;

/* Defaults (no window, default tuning for every qubit count). */
KATE_API kate_status kate_batch_options_default(kate_batch_options* opt);
/* The autotuner: for each qubit count present in `circuits`, times
 * candidate plans of a sample of those circuits on `device` (fusion x
 * max_gates, then group_qubits, then coalesce, then, for complex64 states
 * kept in device memory, tensor-core blocks) and writes the fastest into
 * opt->tune. */
KATE_API kate_status kate_batch_autotune(const kate_circuit* const* circuits, int count, int precision, int device,
                                         kate_batch_options* opt);
/* opt: nullable (defaults). precision: KATE_C64 or KATE_C128. */
KATE_API kate_status kate_batch_create(const kate_circuit* const* circuits, int count, int precision, int device,
                                       const kate_batch_options* opt, kate_batch** out);
KATE_API kate_status kate_batch_destroy(kate_batch* b);
/* Enqueues one run (one graph launch) on `stream` (NULL: the batch's own). */
KATE_API kate_status kate_batch_run_async(kate_batch* b, void* stream);
/* Waits for the runs; KATE_ECUDA if a dependency wait in the kernel gave up. */
KATE_API kate_status kate_batch_synchronize(kate_batch* b);
/* Runs once and waits. */
KATE_API kate_status kate_batch_run(kate_batch* b);
/* Waits, then copies kate_batch_num_outputs doubles. */
KATE_API kate_status kate_batch_expect_z(kate_batch* b, double* out);
KATE_API kate_status kate_batch_num_outputs(const kate_batch* b, long long* out);
/* info[0] tasks, info[1] pass programs, info[2] arena bytes, info[3] CTAs. */
KATE_API kate_status kate_batch_info(const kate_batch* b, long long* info);
/* Pass programs of the batch that run as tensor-core block passes
 * (kate_batch_tuning.blocks). */
KATE_API kate_status kate_batch_block_programs(const kate_batch* b, long long* out);
/* Per circuit i: programs[i] pass programs, resident_qubits[i] qubits of
 * its device state (0 when it runs in shared memory). Arrays of count. */
KATE_API kate_status kate_batch_circuit_info(const kate_batch* b, int* programs, int* resident_qubits);
/* Average device time of `runs` back-to-back runs (CUDA events). */
KATE_API kate_status kate_batch_time(kate_batch* b, int runs, float* ms);
/* Final state of circuit `circuit` after the last run, 2^n complex128
 * amplitudes (re, im pairs) in the circuit's qubit labels; KATE_EINVAL for a
 * circuit that ran whole in one CTA's shared memory (resident qubits 0 in
 * kate_batch_circuit_info: it keeps no state). For checking a batch's
 * complex64 arithmetic against complex128 (its infidelity); the reference
 * exposes its state as a public member (CPUcode/simulator.hpp:18). */
KATE_API kate_status kate_batch_get_state(kate_batch* b, int circuit, double* out);
/* Host wall time of kate_batch_create in ms, ms[0..3]: planning (host
 * threads), assembly of the task queue, device buffers and uploads, graph
 * capture and instantiation. */
KATE_API kate_status kate_batch_create_times(const kate_batch* b, double* ms);
/* Bytes kate_batch_create copied from host to device (task queue, circuit
 * and program tables, program data, matrices). */
KATE_API kate_status kate_batch_upload_bytes(const kate_batch* b, long long* bytes);

/* ---- serving: a request stream with continuous batching ----
 * Replaces a caller's loop that blocks on `Simulator(circuit).execute()`
 * per request (HIPcode/simulator.hpp:301-353). A server owns an engine
 * thread: kate_server_submit queues a request (12 to 28 qubits, `shots`
 * samples from the seeded splitmix64 stream `seed`) and returns at once;
 * host threads plan it; the engine admits requests in submission order
 * while their states fit `budget_bytes` of device memory, and runs steps,
 * each one launch in which every scheduled request advances by some of its
 * group passes, so requests join and leave between steps. A finished
 * request yields <Z_q> per program label (as kate_sim_expect_z) and its
 * samples (basis-state indices in label order, as kate_sim_sample). */
typedef struct {
    unsigned long long budget_bytes; /* resident states (default 150 GiB) */
    unsigned long long aux_bytes;    /* programs, outputs and sums (default 2 GiB) */
    long long step_tiles;            /* 4096-amplitude tile passes per step (default 65536) */
    int chunk;                       /* cosets per pass task (default 4) */
    int zchunks;                     /* 65536-amplitude chunks per <Z> task (default 4) */
    int schunks;                     /* chunks per sampling task (default 16) */
    int planners;                    /* planning threads (0: hardware concurrency, at most 16) */
    int fusion;                      /* gateFusion width for unfused circuits (1: none) */
    int max_gates;                   /* gates per pass program */
    int step_latency_us;             /* estimated critical path per step (default 1500; <0: no limit) */
    int tensor_blocks;               /* 1: complex64 requests run their passes as 5-qubit tensor-core blocks
                                        (as kate_batch_tuning.blocks; default 0: register-staged programs) */
} kate_server_options;

KATE_API kate_status kate_server_options_default(kate_server_options* opt);
/* opt: nullable (defaults). Allocates the state and aux arenas up front. */
KATE_API kate_status kate_server_create(int precision, int device, const kate_server_options* opt, kate_server** out);
/* Stops the engine after its running step; requests not collected are dropped. */
KATE_API kate_status kate_server_destroy(kate_server* s);
/* Thread-safe; does not wait for the GPU. */
KATE_API kate_status kate_server_submit(kate_server* s, const kate_circuit* c, int shots, uint64_t seed, long long* id);
/* Waits up to timeout_s for request id; KATE_ETIMEDOUT if it is not done.
 * On success writes nqbits, z (nqbits doubles), samples (shots entries) and
 * times (3 doubles: submitted, admitted, done; seconds since the server
 * started), each nullable, and forgets the request. */
KATE_API kate_status kate_server_wait(kate_server* s, long long id, double timeout_s, int* nqbits, double* z,
                                      uint64_t* samples, double* times);
/* out[12]: submitted, completed, live, queued, steps, resident bytes, peak resident bytes, failed, then the
 * engine thread's microseconds in admission, step building, step kernels (launch to completion) and result
 * collection. */
KATE_API kate_status kate_server_stats(const kate_server* s, long long* out);
/* Seconds since the server started (the clock of kate_server_wait's times). */
KATE_API kate_status kate_server_now(const kate_server* s, double* t);

#ifdef __cplusplus
}
#endif

#endif /* KATE_B200_H */
