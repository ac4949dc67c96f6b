// engine.h — internal declarations shared by the host planner/ABI (C++) and
// the CUDA kernels of the B200 state-vector engine.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/aleph_b200.h"

namespace ab {

// ---------------------------------------------------------------------------
// Device ops. A gate is lowered to one Op; passes apply ordered Op lists.
// ---------------------------------------------------------------------------
enum OpType : uint8_t {
  OP_1Q = 1,      // dense 2x2 on one target (coef: 4 complex, row-major)
  OP_2Q = 2,      // dense 4x4 on two targets, q[0] = matrix MSB (coef: 16 complex)
  OP_X = 3,       // Pauli-X permutation on one target (no arithmetic)
  OP_CPHASE = 4,  // amp *= coef[0] where every bit of `mask` is 1 (Z, S, T, Phase, CZ, CCZ, ...)
  OP_DIAG = 5,    // amp *= coef[idx], idx = bits of q[0..nq) MSB-first (nq <= 3)
  OP_POLY = 6,    // DiagonalPhase: amp *= exp(i*phi(x)), terms [mask, mask+aux)
  OP_KQ = 7,      // dense 2^k x 2^k, k = nq (3..5), q MSB-first (coef: 4^k complex)
  OP_NEG = 8,     // amp = -amp where every bit of `mask` is 1 (CZ, CCZ, Z fast path)
};

struct Op {
  uint8_t type;
  uint8_t nq;      // target count in q[]
  uint8_t a, b;    // tile slots of q[0] / q[1] (tile kernel); see TilePass
  uint8_t q[6];    // global target qubits, MSB-first
  uint8_t creg;    // tile kernel: control / mask bits that are register qubits (R-bit mask)
  uint8_t dsrc;    // tile kernel, OP_DIAG: bit i set -> table bit i comes from register slot q[3+i]
  uint64_t ctrl;   // global control mask: op acts where (x & ctrl) == ctrl
                   // (tile kernel: only the bits outside the register qubits)
  uint64_t mask;   // OP_CPHASE / OP_NEG: qubit mask (tile kernel: bits outside the
                   // register qubits; the register part is in creg); OP_POLY: first term
  uint32_t coef;   // offset into the coefficient pool (complex elements)
  uint32_t aux;    // OP_POLY: term count
};
static_assert(sizeof(Op) == 40, "Op layout");

// Diagonal-phase polynomial tables (OP_POLY), device-resident per plan.
struct PolyTables {
  const double* angle;
  const uint32_t* cond_off;
  const uint32_t* cond_cnt;
  const uint64_t* conds;
};

// Warp-tile pass: lanes hold qubits 0..4 (one amplitude per lane), each
// thread holds 2^R amplitudes over the R "register" qubits hq[0..R).
// Slot numbering of Op::a/b: 0..4 = lane bit (= qubit), 5+j = register bit j.
struct TilePass {
  uint32_t n;
  uint32_t R;
  uint32_t hq[5];
  uint32_t op_begin;
  uint32_t op_count;
  uint32_t occupancy;  // resident 128-thread blocks per SM the kernel variant targets (2..4; 0 = default)
};

// Tensor-core dense-block pass (TC32): a 2^6 x 2^6 complex matrix on the
// qubits bq[0..6) (ascending; bq[j] = bit j of the block row index), with
// diagonal ops applied before (pre) and after (post) the block product.
struct BlockPass {
  uint32_t n;
  uint32_t bq[6];
  uint32_t mat;        // offset of the split BF16 operand images in the block pool (bytes)
  uint32_t pre_begin, pre_count, post_begin, post_count;
  // some post op is a phase that folds into per-column factors (a corner
  // phase with at most one block qubit, or a one-qubit diagonal on a
  // non-block qubit with no block controls): the kernel variant that folds
  uint32_t fold;
};

// Kind 6 is the renormalisation that follows a tensor-core stream (pass records only).
enum PassKind : uint8_t {
  PASS_TILE = 1,
  PASS_SMEM = 2,
  PASS_KQ = 3,
  PASS_MEASURE = 4,
  PASS_BLOCK = 5,
  PASS_PERMUTE = 7,
};

constexpr uint32_t kMaxQubits = 40;

struct Pass {
  PassKind kind;
  TilePass tile;       // PASS_TILE (also op range for PASS_SMEM / PASS_KQ)
  BlockPass block;     // PASS_BLOCK
  uint32_t qubit;      // PASS_MEASURE
  // PASS_PERMUTE: an involution of the qubit positions; the pass maps
  // psi(j) -> psi(sigma(j)), sigma(j) moving bit q of j to position sigma[q]
  uint8_t sigma[kMaxQubits];
  uint32_t record;     // instruction index (errors, outcome slot)
  uint32_t gates;      // gates consumed (stats / cost model)
  // cost-model features: non-diagonal ops on lane qubits, all non-diagonal ops, diagonal ops
  uint32_t lane_ops = 0, dense_ops = 0, diag_ops = 0;
  uint32_t fma_per_amp = 0;  // tile pass: real multiply-adds per amplitude
};

// ---------------------------------------------------------------------------
// Host-side lowered gate (validated) and plans.
// ---------------------------------------------------------------------------
struct Lowered {
  Op op;
  std::vector<double> coef;  // complex pairs (re, im)
  uint64_t nondiag;          // qubits the op acts on non-diagonally
  uint64_t diag;             // qubits the op reads only diagonally (controls, diagonal targets)
  uint32_t record;           // source instruction index
  bool is_measure = false;
  uint32_t measure_qubit = 0;
  // a qubit-permutation pass (an involution of the positions, see Pass::sigma);
  // `gates` SWAP records were absorbed into it
  bool is_permute = false;
  std::vector<uint8_t> sigma;
  uint32_t gates = 0;
  // OP_POLY terms (DiagonalPhase): angle, condition count, condition masks
  std::vector<double> poly_angle;
  std::vector<uint32_t> poly_cnt;
  std::vector<uint64_t> poly_conds;
};

struct Plan {
  std::vector<Pass> passes;
  std::vector<Op> ops;
  std::vector<double> coef;  // complex pairs
  // OP_POLY tables
  std::vector<double> poly_angle;
  std::vector<uint32_t> poly_off, poly_cnt;
  std::vector<uint64_t> poly_conds;
  // TC32 split-BF16 block operand images (bytes), one 64 KiB image per block
  std::vector<uint8_t> block_images;
  uint32_t n_measures = 0;
  // TC32: renormalise the state after the block passes. Off for plans that
  // run on one tile group of an out-of-core state, whose norm is not 1.
  bool renormalize = true;
};

struct PlanOptions {
  uint32_t tile_r = 5;          // register qubits per warp tile
  uint32_t smem_max_n = 12;     // states with n <= this run as one shared-memory pass
  bool tensor_blocks = false;   // TC32: fuse into 6-qubit dense blocks
  uint32_t block_k = 6;
  bool block_window_search = true;  // TC32: also try every 6-qubit window per pass
  uint32_t tile_occupancy = 0;      // tile kernel variant: 128-thread blocks per SM (0 = 2)
  bool relabel_swaps = true;        // SWAPs relabel qubits; one permutation pass settles the map
  bool renormalize = true;          // TC32: rescale to norm 1 after a stream's block passes
  bool pair_fusion = true;          // tile passes: a two-qubit gate and its one-qubit neighbours as one 4x4
};

// ---------------------------------------------------------------------------
// Engine objects.
// ---------------------------------------------------------------------------
struct State {
  uint32_t n = 0;
  int precision = ALEPH_B200_F64;
  void* amps = nullptr;   // double2[2^n] or float2[2^n]
  size_t bytes = 0;
};

struct Scratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};

struct Handle {
  int device = 0;
  int precision = ALEPH_B200_F64;
  uint32_t qubit_cap = 33;
  cudaStream_t stream = nullptr;
  uint64_t rng_state[2] = {0, 0};
  aleph_b200_error_info err{};
  std::string err_msg;
  aleph_b200_stats stats{};
  PlanOptions opts;
  int sm_count = 148;
  // out-of-core runs: cap on the qubits of one device tile group (0: the
  // most that `depth` buffers fit in half of the free device memory)
  uint32_t paged_local_max = 0;
  // device scratch (grown on demand, freed with the handle)
  Scratch reduce;    // reduction partials
  Scratch plan_buf;  // uploaded plan tables
  Scratch sample;    // sampling tables
  Scratch status;    // device status words (measure outcomes, error flags)
  // freed state buffers kept for reuse by the next allocate of the same size
  // (stream-ordered: reuse runs after the kernels that used the buffer)
  std::vector<Scratch> state_pool;
  // per-pass timing (record_passes)
  bool record_passes = false;
  std::vector<cudaEvent_t> events;
  std::vector<aleph_b200_pass_record> records;
  // batched QAOA sweep: device buffers, pinned staging and the captured graph
  struct Qaoa {
    Scratch dev;           // sets | order | edges | angles | out | counter
    Scratch state;         // per-CTA state slices (streamed sets)
    Scratch cuts;          // per-CTA cut(z) slices
    void* host_in = nullptr;   // pinned staging of the device input region
    void* host_out = nullptr;  // pinned staging of the results
    size_t host_in_bytes = 0, host_out_bytes = 0;
    cudaGraphExec_t exec = nullptr;
    uint64_t key[6] = {0, 0, 0, 0, 0, 0};  // layout the graph was captured for
  } qaoa;
};

// Accepted |sum |a|^2 - 1| of a state before readout: the FP64 drift budget
// sqrt(N) * AMPLITUDE_TOL (crates/aleph-sv/src/measure.rs:23-33), and for FP32
// states the reference FP32 backend's FP32_NORM_TOL = 1e-4
// (crates/aleph-sv/src/fp32_measure.rs:20-23).
inline __host__ __device__ double norm_tolerance(uint64_t len, int precision) {
  return precision == ALEPH_B200_F64 ? sqrt((double)len) * 1e-10 : 1e-4;
}

// kernels_*.cu entry points (host wrappers; all launch on `stream`)
cudaError_t launch_init_zero_state(void* amps, uint32_t n, int precision, cudaStream_t s);
// dev_error: set to ALEPH_B200_DEVICE_FAILURE by a pass kernel whose bounded copy wait expires.
cudaError_t launch_tile_pass(void* amps, int precision, const TilePass& p, const Op* ops, const void* coef,
                             PolyTables poly, int* dev_error, int sm_count, cudaStream_t s);
cudaError_t launch_smem_pass(void* amps, int precision, uint32_t n, const Op* ops, uint32_t op_count,
                             const void* coef, PolyTables poly, cudaStream_t s);
cudaError_t launch_kq_pass(void* amps, int precision, uint32_t n, const Op* op_dev, const Op& op_host,
                           const void* coef, cudaStream_t s);
cudaError_t launch_block_pass(void* amps, const BlockPass& p, const uint8_t* images, const Op* ops,
                              const void* coef, PolyTables poly, int* dev_error, int sm_count, cudaStream_t s);
// amps *= 1 / sqrt(*norm2) (norm2 in device memory).
cudaError_t launch_rescale(void* amps, int precision, uint32_t n, const double* norm2, cudaStream_t s);
cudaError_t launch_renormalize(void* amps, int precision, uint32_t n, double* partials, uint32_t nblocks, double* out2,
                               cudaStream_t s);
cudaError_t launch_convert(const void* src, int src_prec, void* dst, int dst_prec, uint64_t count, cudaStream_t s);
// In-place qubit-permutation pass: psi(j) -> psi(sigma(j)) for an involution
// sigma of the n qubit positions (sigma[sigma[q]] == q).
cudaError_t launch_permute_pass(void* amps, int precision, uint32_t n, const uint8_t* sigma, int sm_count,
                                cudaStream_t s);
// Splits the position permutation pi (bit q of an index moves to pi[q]) into
// involutions applied in order: psi o pi = P_last ... P_first psi, where a
// pass P_sigma maps psi(j) -> psi(sigma(j)). At most two; none for the identity.
std::vector<std::vector<uint8_t>> split_into_involutions(const std::vector<uint32_t>& pi);

// readout (kernels_readout.cu)
// partial sums: out[0] = sum |a|^2, out[1] = count of non-finite |a|^2
cudaError_t launch_norm(const void* amps, int precision, uint32_t n, double* partials, uint32_t nblocks,
                        double* out2, cudaStream_t s);
cudaError_t launch_measure_pass(void* amps, int precision, uint32_t n, uint32_t qubit, double* partials,
                                uint32_t nblocks, const double* uniforms, uint32_t n_uniforms, int32_t* status,
                                uint8_t* outcome_slot, cudaStream_t s);
cudaError_t launch_expectation(const void* amps, int precision, uint32_t n, uint64_t xmask, uint64_t zmask,
                               uint32_t ny, double* partials, uint32_t nblocks, double* out3, cudaStream_t s);
// Up to MAX_TERMS Pauli strings with the same X/Y positions (xmask), each with
// its Z/Y positions and number of Y factors: evaluated in one sweep.
struct PauliGroup {
  static constexpr int MAX_TERMS = 16;
  uint64_t xmask;
  uint32_t count;
  uint64_t zmask[MAX_TERMS];
  uint32_t ny[MAX_TERMS];
};
// out: [sum |a|^2, non-finite count, Re <P_0>, ..., Re <P_15>] (2 + MAX_TERMS doubles)
cudaError_t launch_pauli_group(const void* amps, int precision, uint32_t n, const PauliGroup& g, double* partials,
                               uint32_t nblocks, double* out, cudaStream_t s);
cudaError_t launch_probabilities(const void* amps, int precision, uint32_t n, const uint32_t* qubits_dev, uint32_t k,
                                 double* partials, uint32_t nblocks, double* out, double* norm_out, cudaStream_t s);
uint32_t reduce_blocks(uint32_t n, int sm_count);

// learned planner cost model (kernels_mlp.cu): F -> H -> H -> H -> 1 MLP
size_t mlp_param_count(int F, int H);
cudaError_t mlp_forward(const float* params, const float* X, float* acts, int B, int F, int H, cudaStream_t s);
cudaError_t mlp_backward(const float* params, const float* X, const float* acts, const float* y, float* grads,
                         float* dbuf, float* loss_dev, int B, int F, int H, cudaStream_t s);
cudaError_t mlp_adam(float* params, const float* grads, float* m, float* v, size_t n, float lr, int step,
                     cudaStream_t s);

// batched QAOA sweep (kernels_qaoa.cu): sets with n <= qaoa_smem_max_n run in
// shared memory; larger ones stream through per-CTA slices of slice_amps.
uint32_t qaoa_smem_max_n(int precision);
int qaoa_ctas_per_sm(int precision);
cudaError_t launch_qaoa_sweep(int precision, const aleph_b200_qaoa_set* sets, const uint32_t* edges,
                              const double* angles, const uint32_t* order, uint32_t* next, double* out,
                              void* scratch, uint8_t* cuts, uint64_t slice_amps, uint32_t n_sets, uint32_t p,
                              int grid, cudaStream_t s);

// FP64 issue rate (kernels_peak.cu): DFMA chains only, no memory traffic
cudaError_t launch_dfma_peak(double* out, uint32_t blocks, uint32_t iters, cudaStream_t s);
double dfma_per_launch(uint32_t blocks, uint32_t iters);

// sampling (kernels_sample.cu)
// CUMULATIVE: shots in the rounding guard band are re-resolved against the
// exact sequential prefix sum up to this n; the count goes to status[2].
constexpr uint32_t kExactCumulativeMaxN = 28;
size_t sample_scratch_bytes(uint32_t n, int mode, uint32_t shots);
cudaError_t launch_sample(const void* amps, int precision, uint32_t n, uint32_t shots, int mode, const void* variates_dev,
                          uint64_t* out_dev, void* scratch, size_t scratch_bytes, int32_t* status, int sm_count,
                          cudaStream_t s);
// Fixed device buffer of aleph_b200_sample_cumulative_noalloc: a file-scope
// __device__ array of this many bytes; its address is looked up with
// cudaGetSymbolAddress, with the target device current.
constexpr size_t kFixedSampleScratchBytes = (size_t)8 << 20;
cudaError_t fixed_sample_scratch_address(void** out);

// Split-BF16 hi/lo operand images of a 128x128 real matrix (kernels_block.cu), 64 KiB.
void build_block_image(const double* W, uint8_t* out);
constexpr uint32_t kBlockImageBytes = 65536;

// planner (planner.cpp)
// tiled: the gate is one of a TiledBlock's gates, validated as the
// reference's tiled executor does (fixed-size 2x2 / 4x4 matrix, no
// unitarity check)
// Gate::matrix as a dense row-major complex matrix (interleaved re, im),
// dim 2, 4 or 8 in *dim; UnitaryKq is rejected (it has no fixed-size matrix).
int gate_matrix_dense(const aleph_b200_instr& g, const double* pool, uint64_t pool_len, double* out, int* dim,
                      aleph_b200_error_info* e);
int lower_gate(const aleph_b200_instr& g, uint32_t n, const double* pool, uint64_t pool_len, Lowered* out,
               aleph_b200_error_info* err, bool tiled = false);
int lower_diagonal_phase(const aleph_b200_phase_term* terms, uint64_t n_terms, const uint64_t* conds, uint64_t n_conds,
                         Lowered* out, aleph_b200_error_info* err);
const char* gate_name(uint32_t kind);
int build_plan(const std::vector<Lowered>& ops, uint32_t n, const PlanOptions& o, Plan* plan);

}  // namespace ab
