/*
 * aleph_b200.h — C ABI of the B200-native dense state-vector engine.
 *
 * The entry points mirror aleph's `Backend` trait
 * (crates/aleph-backend/src/lib.rs:86-163) so that a host binding (Rust FFI,
 * ctypes, pybind) can stand in for the `sv` / `cuda` backends:
 *
 *   Backend::allocate             -> aleph_b200_allocate
 *   Backend::apply_gate           -> aleph_b200_apply_gate
 *   Backend::apply_diagonal_phase -> aleph_b200_apply_diagonal_phase
 *   Backend::apply_tiled_block    -> aleph_b200_apply_gate_stream (TILED_BLOCK record)
 *   Backend::unpermute_state      -> aleph_b200_unpermute
 *   Backend::measure              -> aleph_b200_measure
 *   Backend::sample               -> aleph_b200_sample / aleph_b200_sample_seeded
 *   Backend::expectation_value    -> aleph_b200_expectation
 *   expectation_pauli_sum         -> aleph_b200_expectation_sum
 *   Backend::probabilities        -> aleph_b200_probabilities
 *   run / run_with_outcomes       -> aleph_b200_apply_gate_stream
 *     (crates/aleph-backend/src/lib.rs:182-245)
 *   CudaSvBackend::run_paged[_overlapped] -> aleph_b200_paged_run
 *     (crates/aleph-cuda/src/sv/paged.rs:138-276)
 *
 * Every function returns an aleph_b200_status (0 = OK). Non-zero codes map
 * 1:1 onto the variants of `BackendError` (crates/aleph-backend/src/lib.rs:22-74);
 * the message and payload of the last error are available through
 * aleph_b200_last_error / aleph_b200_last_error_info. The engine never aborts
 * the process and never traps the GPU.
 *
 * Plain C types only: pointers, sizes, POD structs. No framework types.
 */
#ifndef ALEPH_B200_H
#define ALEPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALEPH_B200_ABI_VERSION 1

/* ---- status codes: BackendError variants (crates/aleph-backend/src/lib.rs:22-74) ---- */
typedef enum aleph_b200_status {
  ALEPH_B200_OK = 0,
  ALEPH_B200_DEVICE_FAILURE = 1,          /* DeviceFailure(String)                 */
  ALEPH_B200_QUBIT_OUT_OF_RANGE = 2,      /* QubitOutOfRange { qubit, num_qubits } */
  ALEPH_B200_DUPLICATE_QUBIT = 3,         /* DuplicateQubit { qubit }              */
  ALEPH_B200_ARITY_MISMATCH = 4,          /* ArityMismatch { kind, expected, got } */
  ALEPH_B200_UNSUPPORTED_GATE = 5,        /* UnsupportedGate { kind }              */
  ALEPH_B200_UNSUPPORTED_INSTRUCTION = 6, /* UnsupportedInstruction { kind }       */
  ALEPH_B200_SYMBOLIC_PARAM = 7,          /* SymbolicParam                         */
  ALEPH_B200_NON_FINITE_PARAM = 8,        /* NonFiniteParam { kind }               */
  ALEPH_B200_NON_UNITARY_MATRIX = 9,      /* NonUnitaryMatrix { deviation }        */
  ALEPH_B200_EMPTY_CIRCUIT = 10,          /* EmptyCircuit                          */
  ALEPH_B200_DEGENERATE_MEASUREMENT = 11, /* DegenerateMeasurement { qubit, p }    */
  ALEPH_B200_TOO_MANY_QUBITS = 12,        /* TooManyQubits { requested, limit }    */
  ALEPH_B200_INVALID_PAULI_STRING = 13,   /* InvalidPauliString { reason }         */
  ALEPH_B200_INVALID_STATE = 14,          /* InvalidState { reason }               */
  ALEPH_B200_OPTIMIZATION = 15,           /* Optimization(PassError)               */
  ALEPH_B200_INVALID_ARGUMENT = 16        /* ABI misuse: null pointer, bad enum    */
} aleph_b200_status;

/* ---- gate kinds: the `Gate` enum, declaration order (crates/aleph-core/src/gate/kinds.rs:12-107) ---- */
typedef enum aleph_b200_kind {
  ALEPH_GATE_H = 0,
  ALEPH_GATE_X = 1,
  ALEPH_GATE_Y = 2,
  ALEPH_GATE_Z = 3,
  ALEPH_GATE_S = 4,
  ALEPH_GATE_SDG = 5,
  ALEPH_GATE_T = 6,
  ALEPH_GATE_TDG = 7,
  ALEPH_GATE_RX = 8,         /* params[0] = theta                       */
  ALEPH_GATE_RY = 9,
  ALEPH_GATE_RZ = 10,
  ALEPH_GATE_PHASE = 11,
  ALEPH_GATE_U3 = 12,        /* params = (theta, phi, lambda)           */
  ALEPH_GATE_CNOT = 13,      /* qubits = [control, target]              */
  ALEPH_GATE_CZ = 14,
  ALEPH_GATE_SWAP = 15,
  ALEPH_GATE_ISWAP = 16,
  ALEPH_GATE_ISWAPDG = 17,
  ALEPH_GATE_CRX = 18,       /* qubits = [control, target]              */
  ALEPH_GATE_CRY = 19,
  ALEPH_GATE_CRZ = 20,
  ALEPH_GATE_TOFFOLI = 21,   /* qubits = [c0, c1, target]               */
  ALEPH_GATE_CCZ = 22,
  ALEPH_GATE_UNITARY1Q = 23, /* 4 complex (row-major) at data_offset    */
  ALEPH_GATE_UNITARY2Q = 24, /* 16 complex, qubits[0] = matrix MSB      */
  ALEPH_GATE_UNITARYKQ = 25, /* aux = k (2..5), 4^k complex, MSB-first  */
  ALEPH_GATE_UNITARY1QDIAG = 26, /* 2 complex diagonal entries          */
  ALEPH_GATE_UNITARY2QDIAG = 27, /* 4 complex diagonal entries          */
  /* non-gate instructions (crates/aleph-ir/src/instruction.rs:13-34) */
  ALEPH_INSTR_MEASURE = 100,        /* qubits[0] = qubit, aux = clbit           */
  ALEPH_INSTR_RESET = 101,          /* rejected: UnsupportedInstruction "reset" */
  ALEPH_INSTR_BARRIER = 102,        /* no-op; data_offset = mask of its qubits  */
  ALEPH_INSTR_DIAGONAL_PHASE = 103, /* terms [data_offset, data_offset+data_len) */
  ALEPH_INSTR_TILED_BLOCK = 104     /* aux = tile_bits; the next data_len records are its gates */
} aleph_b200_kind;

/* One instruction of the flattened aleph-ir gate stream. `GateInstance`
 * (crates/aleph-core/src/gate/instance.rs:56-61) is {gate, qubits, controls};
 * qubits are in the gate's operand order (qubits[0] = matrix MSB). */
typedef struct aleph_b200_instr {
  uint32_t kind;          /* aleph_b200_kind                                        */
  uint32_t num_qubits;    /* entries used in qubits[]                               */
  uint32_t num_controls;  /* entries used in controls[]                             */
  uint32_t aux;           /* MEASURE: clbit; UNITARYKQ: k; TILED_BLOCK: tile_bits   */
  uint32_t qubits[8];
  uint32_t controls[8];
  double params[3];
  uint64_t data_offset;   /* matrix pool offset in complex elements / first term    */
  uint64_t data_len;      /* complex elements / terms / TILED_BLOCK gate count      */
} aleph_b200_instr;

/* One `PhaseTerm` (crates/aleph-ir/src/diagonal_phase.rs:20-26): adds `angle`
 * to the phase of |x> when parity(mask & x) is odd for every mask in
 * cond_pool[cond_offset .. cond_offset + cond_count). */
typedef struct aleph_b200_phase_term {
  double angle;
  uint32_t cond_offset;
  uint32_t cond_count;
} aleph_b200_phase_term;

/* Side tables of a gate stream. Any pointer may be NULL when its count is 0. */
typedef struct aleph_b200_pools {
  const double* matrix_pool;           /* interleaved (re, im) complex */
  uint64_t matrix_pool_len;            /* in complex elements          */
  const aleph_b200_phase_term* terms;
  uint64_t n_terms;
  const uint64_t* cond_pool;
  uint64_t n_conds;
} aleph_b200_pools;

typedef enum aleph_b200_precision {
  ALEPH_B200_F64 = 0,  /* complex128 state, FP64 arithmetic                         */
  ALEPH_B200_F32 = 1,  /* complex64 state, FP32 CUDA-core arithmetic                */
  ALEPH_B200_TC32 = 2  /* complex64 state, fused 6-qubit blocks on tcgen05 tensor
                          cores with split-BF16x3 operands and FP32 accumulation   */
} aleph_b200_precision;

typedef enum aleph_b200_sample_mode {
  /* one uint64 word per shot, Vose alias table
     (crates/aleph-sv/src/sampling.rs:93-198); the reference's shots >= 2 path */
  ALEPH_B200_SAMPLE_ALIAS = 0,
  /* one double in [0,1) per shot, inverse CDF with cumulative_index semantics
     (crates/aleph-sv/src/sampling.rs:59-91); the reference's shots <= 1 path */
  ALEPH_B200_SAMPLE_CUMULATIVE = 1,
  /* the reference's own rule: ALIAS when shots >= 2, CUMULATIVE otherwise
     (crates/aleph-sv/src/measure.rs:109-124); `variates` then holds uint64
     words for ALIAS, or one double for CUMULATIVE */
  ALEPH_B200_SAMPLE_AUTO = 2
} aleph_b200_sample_mode;

typedef enum aleph_b200_pauli { ALEPH_PAULI_I = 0, ALEPH_PAULI_X = 1, ALEPH_PAULI_Y = 2, ALEPH_PAULI_Z = 3 } aleph_b200_pauli;

typedef struct aleph_b200_handle aleph_b200_handle;
typedef struct aleph_b200_state aleph_b200_state;

/* Payload of the last error (fields not used by a variant are zero). */
typedef struct aleph_b200_error_info {
  int32_t status;
  uint32_t qubit;       /* QubitOutOfRange, DuplicateQubit, DegenerateMeasurement */
  uint32_t num_qubits;  /* QubitOutOfRange                                        */
  uint32_t expected;    /* ArityMismatch                                          */
  uint32_t got;         /* ArityMismatch                                          */
  uint32_t requested;   /* TooManyQubits                                          */
  uint32_t limit;       /* TooManyQubits                                          */
  uint32_t instruction; /* index of the failing record in a gate stream           */
  double value;         /* NonUnitaryMatrix deviation / DegenerateMeasurement p   */
  char kind[32];        /* gate / instruction name (Gate::name, kinds.rs:156-186) */
} aleph_b200_error_info;

/* ---- lifecycle ---- */

/* Replaces NaiveSvBackend::with_seed / CudaSvBackend::new
 * (crates/aleph-sv/src/backend.rs:36-42, crates/aleph-cuda/src/sv/backend.rs:94-129).
 * Binds `device`, creates one stream and the per-handle RNG seeded with `seed`. */
int aleph_b200_create(uint64_t seed, int device, int precision, aleph_b200_handle** out);
int aleph_b200_destroy(aleph_b200_handle* h);
/* Qubit cap of `allocate` (MAX_NAIVE_QUBITS analogue, backend.rs:11,46-49).
 * Default: 33 (F64) / 34 (F32, TC32). */
int aleph_b200_set_qubit_cap(aleph_b200_handle* h, uint32_t cap);

/* ---- Backend::allocate (crates/aleph-sv/src/backend.rs:61-72): |0...0> ---- */
int aleph_b200_allocate(aleph_b200_handle* h, uint32_t num_qubits, aleph_b200_state** out);
int aleph_b200_free_state(aleph_b200_handle* h, aleph_b200_state* st);
int aleph_b200_num_qubits(const aleph_b200_state* st, uint32_t* out);
/* Puts an allocated state back to |0...0> on the device (the state a fresh
 * Backend::allocate returns), so one allocation can serve many runs. */
int aleph_b200_reset_state(aleph_b200_handle* h, aleph_b200_state* st);

/* ---- Backend::apply_gate (crates/aleph-sv/src/backend.rs:74-152) ---- */
int aleph_b200_apply_gate(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_instr* gate,
                          const double* matrix_pool, uint64_t matrix_pool_len);

/* ---- run_with_outcomes (crates/aleph-backend/src/lib.rs:211-245) ----
 * Validates the whole stream first (first invalid record -> its error, state
 * untouched), then plans and launches it. MEASURE records draw one uniform
 * from `measure_uniforms` per non-degenerate measurement, in order; with
 * measure_uniforms == NULL the handle's RNG supplies them. Outcomes (0/1) are
 * written to `outcomes` in record order; `*n_outcomes` receives their count. */
int aleph_b200_apply_gate_stream(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_instr* instrs,
                                 uint64_t count, const aleph_b200_pools* pools, const double* measure_uniforms,
                                 uint64_t n_uniforms, uint8_t* outcomes, uint64_t outcomes_cap,
                                 uint64_t* n_outcomes);

/* ---- compiled plans: CudaExecutionPlan::compile / execute
 * (crates/aleph-cuda/src/execution.rs:57-78,183) ----
 * aleph_b200_compile validates and plans a record stream for a
 * `num_qubits`-qubit register of this handle once; the plan tables are
 * uploaded to device memory at the first execute and stay resident.
 * aleph_b200_execute then applies the plan to `st` (same qubit count) with
 * the semantics of aleph_b200_apply_gate_stream. A plan belongs to the handle
 * that compiled it; calls on one handle are stream-ordered. */
typedef struct aleph_b200_plan aleph_b200_plan;
int aleph_b200_compile(aleph_b200_handle* h, uint32_t num_qubits, const aleph_b200_instr* instrs, uint64_t count,
                       const aleph_b200_pools* pools, aleph_b200_plan** out);
int aleph_b200_execute(aleph_b200_handle* h, aleph_b200_state* st, aleph_b200_plan* plan,
                       const double* measure_uniforms, uint64_t n_uniforms, uint8_t* outcomes, uint64_t outcomes_cap,
                       uint64_t* n_outcomes);
int aleph_b200_plan_free(aleph_b200_handle* h, aleph_b200_plan* plan);

/* ---- batched QAOA Max-Cut sweep ----
 * Evaluates <C> = <psi|H_C|psi>, H_C = sum_edges 1/2 (I - Z_i Z_j)
 * (maxcut_pauli_sum, crates/aleph-ir/src/ansatz.rs:100-117), for many
 * parameter sets at once; set k's state is the build_qaoa circuit
 * (ansatz.rs:71-98) on sets[k].num_qubits qubits with the edges
 * edges[2e], edges[2e+1] for e in [edge_offset, edge_offset + num_edges) and
 * the angles angles[2p k .. 2p k + p) (gammas) and angles[2p k + p .. 2p(k+1))
 * (betas). The state precision is the handle's (F64: complex128; F32 and
 * TC32: complex64); <C> is reduced in FP64 either way. All sets run in one
 * persistent launch, replayed as a CUDA graph while the batch layout
 * (counts, sizes) stays the same. Limits: 1 <= num_qubits <= 26, num_edges
 * <= 128, p >= 1. Errors: QubitOutOfRange / DuplicateQubit for a bad edge
 * (the reference's CNOT(i, j) checks), NonFiniteParam, TooManyQubits. */
typedef struct aleph_b200_qaoa_set {
  uint32_t num_qubits;
  uint32_t num_edges;
  uint64_t edge_offset; /* in (u, v) pairs */
} aleph_b200_qaoa_set;
int aleph_b200_qaoa_sweep(aleph_b200_handle* h, uint32_t p, const aleph_b200_qaoa_set* sets, uint32_t n_sets,
                          const uint32_t* edges, uint64_t n_edge_pairs, const double* angles, double* expectations);

/* ---- Backend::apply_diagonal_phase (crates/aleph-sv/src/kernels/diagonal_phase.rs:74-97) ---- */
int aleph_b200_apply_diagonal_phase(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_phase_term* terms,
                                    uint64_t n_terms, const uint64_t* cond_pool, uint64_t n_conds);

/* ---- Backend::unpermute_state (crates/aleph-core/src/perm.rs:25-40): perm[logical] = physical ----
 * In place: at most two involution passes, no second state buffer. */
int aleph_b200_unpermute(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* perm, uint32_t n);

/* ---- Backend::measure (crates/aleph-sv/src/measure.rs:41-102) ----
 * `u` is the uniform consumed when both branches are non-degenerate; pass a
 * negative value to draw it from the handle's RNG. *consumed = 1 if it was used. */
int aleph_b200_measure(aleph_b200_handle* h, aleph_b200_state* st, uint32_t qubit, double u, int* outcome,
                       int* consumed);

/* ---- Backend::sample (crates/aleph-sv/src/measure.rs:109-148) ----
 * `variates`: uint64 words (ALIAS) or doubles in [0,1) (CUMULATIVE), one per shot. */
int aleph_b200_sample(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots, int mode, const void* variates,
                      uint64_t* out);
/* Same, with variates drawn from the handle's RNG: ALIAS (one u64 per shot)
 * for 2+ shots on n <= 20, otherwise CUMULATIVE (one double per shot), which
 * covers every n, including those above the alias limit of 28. */
int aleph_b200_sample_seeded(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots, uint64_t* out);

/* CUMULATIVE sampling that allocates nothing. No counterpart in the reference.
 * Same kernels and results as aleph_b200_sample(..., ALEPH_B200_SAMPLE_CUMULATIVE,
 * ...), but all device scratch lives in one fixed 8 MiB buffer per device (no
 * cudaMalloc / cudaFree), for callers that cannot allocate at that point:
 * state vectors that already fill HBM, or latency-bound sampling loops where
 * scratch growth would synchronise the device.
 *  - The buffer is reserved when the first handle on a device is created
 *    (aleph_b200_create loads the module that holds it), before any state is
 *    allocated; each call looks up its address with the handle's device
 *    current, so a device reset by the host program is followed correctly.
 *  - Limit: the scratch of (n, shots) must fit the 8 MiB (n <= 30 fits up to
 *    65536 shots); larger requests return ALEPH_B200_INVALID_ARGUMENT.
 *  - The buffer is shared by all handles on a device: calls that overlap in
 *    time on one device (several host threads, or handles whose streams
 *    run concurrently) race on it; serialise them. Each call synchronises
 *    its handle's stream before it returns. */
int aleph_b200_sample_cumulative_noalloc(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots,
                                         const double* variates, uint64_t* out);

/* ---- Backend::expectation_value (crates/aleph-sv/src/measure.rs:155-233) ---- */
int aleph_b200_expectation(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits,
                           const uint8_t* paulis, uint32_t n_terms, double coefficient, double* out);

/* ---- expectation_pauli_sum (crates/aleph-backend/src/lib.rs:422-432) ----
 * out = sum over terms k of coefficients[k] * Re <psi| P_k |psi>, where P_k is
 * the Pauli string qubits[offsets[k] .. offsets[k+1]) with codes
 * paulis[same range] (offsets has n_terms + 1 entries). The reference loops
 * expectation_value over the terms; here the terms that share their X/Y
 * positions are evaluated together, up to 16 per sweep of the state, and all
 * results come back with one host synchronisation. Each term's value agrees
 * with what aleph_b200_expectation returns for it to rounding (the same
 * reduction order). Errors are the reference
 * loop's: none for n_terms = 0; otherwise the state norm first, then each
 * term's coefficient, qubit range and duplicates in term order.
 * term_values (optional, n_terms doubles) receives each coefficients[k] * <P_k>. */
int aleph_b200_expectation_sum(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits,
                               const uint8_t* paulis, const uint64_t* offsets, const double* coefficients,
                               uint64_t n_terms, double* out, double* term_values);

/* ---- Backend::probabilities (crates/aleph-sv/src/measure.rs:239-273): qubits[0] = LSB of the output index ---- */
int aleph_b200_probabilities(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits, uint32_t k,
                             double* out);

/* ---- state access (RunResult.statevector(), crates/aleph-py/src/run.rs:71-101) ----
 * Interleaved (re, im) doubles, 2 * 2^n values; FP32 states are widened. */
int aleph_b200_get_amplitudes(aleph_b200_handle* h, aleph_b200_state* st, double* out);
/* A window of the state: amplitudes [first, first + count) as interleaved
 * (re, im) doubles, for states too large to copy whole to the host (an n=33
 * FP64 state is 128 GiB). The same values as the matching slice of
 * aleph_b200_get_amplitudes (CudaSvState::amplitudes_vec,
 * crates/aleph-cuda/src/sv/state.rs:106); a window outside 2^n amplitudes is
 * ALEPH_B200_INVALID_ARGUMENT. */
int aleph_b200_get_amplitude_range(aleph_b200_handle* h, aleph_b200_state* st, uint64_t first, uint64_t count,
                                   double* out);
int aleph_b200_set_amplitudes(aleph_b200_handle* h, aleph_b200_state* st, const double* in);
/* The state's device memory (2^n interleaved complex128, or complex64 for
 * F32/TC32 handles) and its size in bytes, ordered on the handle's stream
 * (aleph_b200_get_stream). For callers that move amplitudes between states or
 * GPUs themselves: the distributed layer's global-qubit exchanges send and
 * receive halves of it over NCCL (DeviceSv::amps_view / amps_view_mut,
 * crates/aleph-cuda/src/dist/mod.rs:49-62). */
int aleph_b200_state_memory(aleph_b200_handle* h, aleph_b200_state* st, void** device_ptr, uint64_t* bytes);

/* Every amplitude times a real factor > 0, on the device. The distributed
 * layer restores the global norm of a TC32 state held as rank slices (each
 * slice runs without the end-of-stream renormalisation) by scaling every
 * slice by 1 / sqrt(sum of the slices' norms). */
int aleph_b200_scale_state(aleph_b200_handle* h, aleph_b200_state* st, double factor);

/* ---- Gate::matrix (crates/aleph-core/src/gate/kinds.rs:213-400) ----
 * The dense matrix of one gate record (dim 2, 4 or 8, row-major, interleaved
 * re/im, MSB-first operand order) into out[2 * dim * dim]; UnitaryKq records
 * are rejected like the reference's Gate::matrix (no fixed-size matrix). */
int aleph_b200_gate_matrix(const aleph_b200_instr* g, const double* matrix_pool, uint64_t pool_len, double* out,
                           int* dim);

/* FP64 sum of |a_i|^2 on the device. */
int aleph_b200_norm_sqr(aleph_b200_handle* h, aleph_b200_state* st, double* out);

/* ---- stream / errors ---- */
int aleph_b200_synchronize(aleph_b200_handle* h);
/* The handle's CUDA stream (a cudaStream_t), on which every kernel of the
 * handle is launched: callers time or order work against it with their own
 * events. */
int aleph_b200_get_stream(const aleph_b200_handle* h, void** stream);
int aleph_b200_last_error(const aleph_b200_handle* h, char* buf, uint64_t len);
int aleph_b200_last_error_info(const aleph_b200_handle* h, aleph_b200_error_info* out);

/* ---- planner tuning (the autotuner's knobs) ----
 * keys: "tile_r" (register qubits per warp tile, 1..5), "smem_max_n" (states
 * with n <= this run as one shared-memory pass, 0..12), "record_passes"
 * (0/1: time every pass of later gate streams with CUDA events),
 * "relabel_swaps" (0/1, default 1: an uncontrolled SWAP of a state larger
 * than smem_max_n relabels qubits instead of moving data, and one or two
 * in-place permutation passes settle the labels at the end of the stream),
 * "paged_local_qubits" (0..40, default 0: the most qubits one device tile
 * group of an out-of-core run may hold; 0 lets free device memory decide),
 * "tile_occupancy" (0 or 2..4: the tile kernel variant, resident 128-thread
 * blocks per SM), "tensor_blocks" (TC32 handles, 0/1), "block_window_search"
 * (0/1), "renormalize" (0/1, default 1: a TC32 gate stream with tensor-core
 * blocks rescales the state to norm 1 at its end; 0 for states that are one
 * slice of a larger state, whose norm is not 1), "pair_fusion" (0/1,
 * default 1: in warp-tile passes a gate on two qubits and the one-qubit
 * gates next to it on those qubits run as one 4x4 when that saves
 * arithmetic). */
int aleph_b200_set_tuning(aleph_b200_handle* h, const char* key, int64_t value);

/* ---- per-pass timing records (training data of the learned fusion planner) ---- */
typedef struct aleph_b200_pass_record {
  uint32_t kind;        /* 1 = CUDA-core tile pass, 2 = shared-memory pass, 3 = dense k-qubit,
                           4 = measurement, 5 = tensor-core dense block, 6 = renormalisation,
                           7 = qubit permutation (relabelled SWAPs, unpermute)             */
  uint32_t gates;       /* gates the pass applied                                          */
  uint32_t n;           /* state qubits                                                    */
  uint32_t nq;          /* entries used in qubits[]                                        */
  uint32_t qubits[8];   /* tile register qubits / block qubits                             */
  uint32_t post_ops;    /* diagonal ops after a block                                      */
  uint32_t lane_ops;    /* tile pass: non-diagonal ops on the lane qubits 0..4 (shuffles)  */
  uint32_t dense_ops;   /* non-diagonal ops the pass applies (a block: the fused gates)    */
  uint32_t diag_ops;    /* diagonal ops the pass applies (phases, CZ-like, DiagonalPhase)  */
  uint32_t variant;     /* kernel variant (tile pass: blocks per SM)                       */
  uint32_t fma_per_amp; /* tile pass: real multiply-adds per amplitude (8 per dense one-qubit
                           op, 16 per dense 4x4, 4 per diagonal phase; controls ignored)   */
  double ms;            /* device time of the pass (CUDA events on the handle's stream)    */
  double bytes;         /* algorithmic HBM bytes of the pass                               */
} aleph_b200_pass_record;
/* The passes the planner makes of a gate stream, without a device (ms = 0):
 * what aleph_b200_compile would launch for a `num_qubits` register of the
 * given precision and tuning. For plan inspection, the autotuner and the
 * learned planner's features. Returns the validation error of the first
 * invalid record, like aleph_b200_compile. */
typedef struct aleph_b200_plan_config {
  int32_t precision;             /* aleph_b200_precision                     */
  uint32_t tile_r;               /* register qubits per warp tile (1..5)     */
  uint32_t smem_max_n;           /* n <= this: one shared-memory pass        */
  uint32_t block_window_search;  /* TC32: also try every 6-qubit window      */
  uint32_t tile_occupancy;       /* tile kernel variant: 0 (default) or 2..4 */
  uint32_t keep_swaps;           /* 1: SWAP records run as gates; 0: relabel */
  uint32_t no_pair_fusion;       /* 1: tile passes apply every gate as given */
} aleph_b200_plan_config;
int aleph_b200_describe_plan(uint32_t num_qubits, const aleph_b200_plan_config* config, const aleph_b200_instr* instrs,
                             uint64_t count, const aleph_b200_pools* pools, aleph_b200_pass_record* out, uint64_t cap,
                             uint64_t* n_passes);
/* Records of the last gate stream run with "record_passes" on; *n = count. */
int aleph_b200_get_pass_records(const aleph_b200_handle* h, aleph_b200_pass_record* out, uint64_t cap,
                                uint64_t* n);

/* ---- the learned fusion planner's cost model: an FP32 MLP ----
 * n_features -> hidden -> hidden -> hidden -> 1 (ReLU hidden layers), trained
 * with MSE loss and Adam by this library's CUDA kernels on pass features and
 * recorded pass times. No counterpart in the reference (its fusion is a
 * greedy heuristic, crates/aleph-ir/src/passes/fuse_kq.rs:268-400).
 * X is row-major n x n_features; y has n entries. */
typedef struct aleph_b200_mlp aleph_b200_mlp;
int aleph_b200_mlp_create(aleph_b200_handle* h, uint32_t n_features, uint32_t hidden, uint64_t seed,
                          aleph_b200_mlp** out);
int aleph_b200_mlp_free(aleph_b200_handle* h, aleph_b200_mlp* m);
/* Parameter count into *count; copies them out (get) and/or replaces them (set). */
int aleph_b200_mlp_params(aleph_b200_handle* h, aleph_b200_mlp* m, float* get, const float* set, uint64_t* count);
int aleph_b200_mlp_predict(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, uint32_t n, float* y_out);
/* Loss and parameter gradients of one batch (n <= 65536), without an update. */
int aleph_b200_mlp_gradients(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, const float* y, uint32_t n,
                             float* grads_out, float* loss_out);
/* Mini-batch Adam for `epochs` passes over the (seed-shuffled) data; the last batch's loss in *final_loss. */
int aleph_b200_mlp_train(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, const float* y, uint32_t n,
                         uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* final_loss);

/* ---- measured FP64 rate (no counterpart in the reference) ----
 * The double-precision FMA rate this device's CUDA cores sustain, in TFLOP/s
 * (2 flops per FMA), measured now by a compute-only kernel on the handle's
 * stream (best of three ~50 ms launches, CUDA events). It is the roofline of
 * the plain FP64 tile passes, which become FMA-bound when many gates fuse. */
int aleph_b200_fp64_rate(aleph_b200_handle* h, double* tflops);

/* ---- launch statistics (execution_counters, crates/aleph-cuda/src/execution.rs:145-165) ---- */
typedef struct aleph_b200_stats {
  uint64_t kernel_launches;   /* engine kernels launched by this handle            */
  uint64_t passes;            /* full-state HBM passes issued by gate streams       */
  uint64_t tile_passes;       /* of which CUDA-core tile passes                     */
  uint64_t block_passes;      /* of which tensor-core dense-block passes            */
  uint64_t gates_planned;     /* gates consumed by the planner                      */
  double algorithmic_bytes;   /* sum of (amplitudes read + written) * bytes/amp     */
  uint64_t h2d_bytes;         /* bytes copied host -> device (plans, variates, ...) */
  uint64_t d2h_bytes;         /* bytes copied device -> host (results, status)      */
  uint64_t guard_band_shots;  /* CUMULATIVE shots whose target fell within the
                                 rounding guard band of a bin boundary of the
                                 parallel prefix sums                              */
  uint64_t guard_band_inexact;/* of those, shots on states above n = 28, which are
                                 not re-resolved against the sequential sum: their
                                 outcome may differ from the sequential CPU scan's
                                 by one bin                                        */
} aleph_b200_stats;
int aleph_b200_get_stats(const aleph_b200_handle* h, aleph_b200_stats* out);
int aleph_b200_reset_stats(aleph_b200_handle* h);

/* ---- out-of-core runs (crates/aleph-cuda/src/sv/paged.rs:138-276) ----
 * The 2^n state lives in pinned host memory, split into 2^(n-m) tiles of
 * 2^m amplitudes (m = tile_qubits low qubits). The gate list is cut into
 * segments whose gates touch few enough high qubits (>= m) that the tiles a
 * segment couples fit the device; each segment gathers every such tile
 * group into device memory (high qubit H[r] -> local qubit m + r), runs the
 * segment there as one compiled plan, and scatters the group back: one read
 * and one write of the host state per segment, copies overlapped with
 * compute over `depth` device buffers (1 = no overlap; 0 = the default 3).
 * Errors as the reference's run_paged: EmptyCircuit for n = 0 and no
 * instructions; InvalidState unless 1 <= tile_qubits < num_qubits;
 * UnsupportedInstruction for measure / reset / diagonal-phase / tiled-block;
 * TooManyQubits when tile_qubits plus the high qubits of one gate exceed
 * what the device holds; then the in-core stream's gate validation. FP64
 * handles keep complex128 tiles, the others complex64 (TC32 segments run
 * their block passes without the final renormalisation). */
typedef struct aleph_b200_paged_state aleph_b200_paged_state;
typedef struct aleph_b200_paged_info {
  uint32_t num_qubits;
  uint32_t tile_qubits;     /* m */
  uint32_t local_qubits;    /* the largest tile group on the device: m + its high qubits */
  uint32_t depth;           /* device buffers in the ring */
  uint64_t segments;        /* sweeps over the host state */
  uint64_t groups;          /* tile groups gathered, computed and scattered */
  uint64_t h2d_bytes, d2h_bytes;
  double seconds;           /* wall time of the run, host allocation excluded */
} aleph_b200_paged_info;
int aleph_b200_paged_run(aleph_b200_handle* h, uint32_t num_qubits, const aleph_b200_instr* instrs, uint64_t count,
                         const aleph_b200_pools* pools, uint32_t tile_qubits, uint32_t depth,
                         aleph_b200_paged_state** out);
int aleph_b200_paged_info_get(const aleph_b200_paged_state* ps, aleph_b200_paged_info* out);
/* Interleaved (re, im) doubles, 2 * 2^n values (PagedSvState::amplitudes_vec, paged.rs:78-87). */
int aleph_b200_paged_get_amplitudes(const aleph_b200_paged_state* ps, double* out);
/* Sum of |a|^2 in FP64 over the host state, block sums Kahan-compensated (PagedSvState::norm_sqr, paged.rs:89-100). */
int aleph_b200_paged_norm_sqr(const aleph_b200_paged_state* ps, double* out);
int aleph_b200_paged_free(aleph_b200_paged_state* ps);
/* Host only, no device: how aleph_b200_paged_run would cut `instrs` for a
 * tile split `tile_qubits` and tile groups of at most `local_qubits` qubits.
 * segment_of[i] (optional, count entries) receives instruction i's segment
 * and position_of[i] (optional) its place in the execution order; barriers
 * get UINT64_MAX in both. Status TOO_MANY_QUBITS when one gate's high qubits
 * do not fit; INVALID_ARGUMENT unless 1 <= tile_qubits < n <= 40 and
 * local_qubits >= tile_qubits. */
int aleph_b200_describe_paged(uint32_t num_qubits, const aleph_b200_instr* instrs, uint64_t count,
                              uint32_t tile_qubits, uint32_t local_qubits, uint64_t* segment_of,
                              uint64_t* position_of, uint64_t* n_segments);

#ifdef __cplusplus
}
#endif
#endif /* ALEPH_B200_H */
