// kernels_block.cu — tensor-core dense-block pass (TC32) for sm_100a.
//
// A pass applies one fused 6-qubit unitary U (64x64 complex, built in FP64 on
// the host) to an FP32 complex state: for every "column" c (an assignment of
// the n-6 other qubits) the 64 amplitudes x_c on the block qubits become
// U x_c. Written as a real GEMM over a tile of 128 columns,
//     D[c][r] = sum_k X[c][k] * W[r][k],
//     X[c] = [Re x_c ; Im x_c]            (128 real values per column),
//     W    = [[Re U, -Im U], [Im U, Re U]] (128 x 128 real),
// so D[c] = [Re U x_c ; Im U x_c]. It runs on the 5th-generation tensor cores
// with split-BF16x3 compensated operands, X = X_hi + X_lo and
// W = W_hi + W_lo (each part BF16), D = X_hi W_hi + X_lo W_hi + X_hi W_lo,
// accumulated in FP32 in TMEM: ~16 significant bits per operand at three BF16
// MMAs per product.
//
// Warp-specialised persistent kernel, one CTA per SM, 14 warps:
//   * warp 12 (TMA): fetches each tile (64 block rows x 128 columns = 64 KiB
//     FP32) with plain (non-multicast) cp.async.bulk copies of its contiguous
//     runs into one of two shared-memory stages (mbarrier transaction counts);
//   * warps 0-3 (converters): thread c takes column c of the staged tile (all
//     64 block rows), splits the real values into BF16 hi/lo and writes them
//     with tcgen05.st into TMEM lane c: the A operand of the MMA lives in
//     tensor memory (two buffers), so shared memory only holds W and the
//     stages;
//   * warp 13 (one thread): issues 3 x 8 tcgen05.mma (A from TMEM, M=128
//     columns; B = W_hi / W_lo from shared memory, N=128, K=16; kind::f16,
//     BF16 in, FP32 accumulate) into one of two TMEM accumulators and commits
//     to mbarriers that free the A buffer and hand the accumulator over;
//   * warps 4-11 (epilogue, two per TMEM lane quarter, one per half of the
//     block rows): tcgen05.ld the accumulator (32x32b: one column
//     per thread), apply the diagonal ops that follow the block (CZ-like sign
//     flips as one 64-bit row mask per thread, other phases per element) and
//     store straight to HBM (16-byte stores of row pairs when the block holds
//     qubit 0, whose rows are then adjacent).
// TMEM: accumulators D0, D1 at columns 0 / 128, A0, A1 at 256 / 384 (hi in the
// first 64 columns, lo in the next 64): all 512 columns.
// Stage layout: the tile's contiguous runs back to back, each followed by a
// pad chosen on the host so that the 32 columns a warp touches at one block
// row fall in distinct shared-memory banks (for blocks on low qubits, whose
// columns are far apart within a run, the columns are chosen above a gap so
// that they index runs, and the pad skews the runs).
// Every wait is bounded; on expiry the CTA records an error code, every role
// leaves its loop, the TMEM is freed and the kernel returns.

#include <cstdint>
#include <cstring>
#include <type_traits>

#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched through the runtime)
#include <cuda_bf16.h>

#include "common.cuh"

namespace ab {

namespace blk {

constexpr int CONV_WARP0 = 0;   // warps 0..3: one per TMEM lane quarter, all 64 block rows
constexpr int CONV_WARPS = 4;
constexpr int EPI_WARP0 = 4;    // warps 4..11: two per TMEM lane quarter, one per half of the block rows
constexpr int EPI_WARPS = 8;
constexpr int TMA_WARP = 12;
constexpr int MMA_WARP = 13;
// 14 warps: with per-SMSP warp slots allocated four at a time this leaves
// 128 registers per thread (18 warps would cap them at 96 and spill)
constexpr int THREADS = 14 * 32;
constexpr int NCOL = 128;                     // columns per tile (MMA M)
constexpr int TILE_AMPS = 64 * NCOL;          // 8192 complex
constexpr int TILE_BYTES = TILE_AMPS * 8;     // 64 KiB FP32 complex
constexpr int MAX_PAD_BYTES = 4096;           // run padding per stage (bank-conflict skew)
constexpr int STAGE_BYTES = TILE_BYTES + MAX_PAD_BYTES;
constexpr int MAX_RUNS = 128;                 // runs per tile (contiguous prefix >= 6 qubits)
constexpr int W_BYTES = 2 * 128 * 128 * 2;    // hi + lo images, 64 KiB
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t TM_D = 0, TM_A = 256;      // accumulators / A operands (128 columns each)
constexpr int MAX_POST = 48;

// shared-memory map (offsets from a 1024-byte aligned base)
constexpr int OFF_W = 0;                                  // B operand: W_hi | W_lo
constexpr int OFF_S = OFF_W + W_BYTES;                    // two FP32 input stages
constexpr int OFF_TAB = OFF_S + 2 * STAGE_BYTES;          // lane-indexed tables
constexpr int TAB_BYTES = NCOL * 4 + NCOL * 8 + MAX_RUNS * 8;
constexpr int OFF_BAR = OFF_TAB + TAB_BYTES;              // mbarriers
constexpr int EPI_STAGE_BYTES = 32 * 8 * 8;               // per epilogue warp: 32 columns x 8 rows
constexpr int OFF_EPI = OFF_BAR + 128;                    // epilogue transposes (blocks on qubits 0..2)
constexpr int SMEM_BYTES = OFF_EPI + EPI_WARPS * EPI_STAGE_BYTES + 1024;  // + alignment slack

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false once about 1 s of wall time has passed
// (kWaitDeadlineNs, %globaltimer) or when another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 0) {
      if (*abort_flag) return false;
      if (globaltimer_ns() - t0 > kWaitDeadlineNs) return false;
    }
  }
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// One tiled tensor copy (no multicast) of the box at coordinates c[0..rank)
// into shared memory, completing `bar`'s transaction count.
__device__ __forceinline__ void tensor_load(uint32_t dst, const CUtensorMap* map, uint32_t rank, const int32_t* c,
                                            uint32_t bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  switch (rank) {
    case 2:
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
              dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(bar)
          : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
          "[%5];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(bar)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
          "[%6];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(bar)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
          "%6}], [%7];" ::"r"(dst),
          "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(bar)
          : "memory");
      break;
  }
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D (TMEM) (+)= A (TMEM, K-major) x B (shared memory descriptor)
__device__ __forceinline__ void tc_mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// tcgen05.ld 32 lanes x 32 bit, 32 consecutive columns per thread.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
// tcgen05.st 32 lanes x 32 bit, 16 consecutive columns per thread.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);         // start address
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;               // stride byte offset
  d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                         // SWIZZLE_128B
  return d;
}
// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both K-major, M=128, N=128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

// Byte offset of element (row r, k) in a K-major SW128 operand image with
// `rows` rows and K = 128 BF16 (two 64-element K regions).
__host__ __device__ __forceinline__ uint32_t sw128_off(uint32_t r, uint32_t k, uint32_t rows) {
  const uint32_t region = k >> 6, kk = k & 63;
  return region * rows * 128 + (r >> 3) * 1024 + (r & 7) * 128 + ((((kk >> 3) ^ (r & 7)) & 7) << 4) + ((kk & 7) << 1);
}

// Two floats to BF16 (round to nearest even) in one instruction: lo -> bits
// 0..15, hi -> bits 16..31.
__device__ __forceinline__ uint32_t bf16x2_bits(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
// Split a pair of floats into packed BF16 hi and lo parts, x = hi + lo to ~16 bits.
__device__ __forceinline__ void split_pair(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  hi = bf16x2_bits(x0, x1);
  const float h0 = __uint_as_float(hi << 16), h1 = __uint_as_float(hi & 0xffff0000u);
  lo = bf16x2_bits(x0 - h0, x1 - h1);
}

}  // namespace blk

// Kernel parameters beyond BlockPass.
struct BlockArgs {
  float2* amps;
  const uint8_t* image;   // W_hi | W_lo, 64 KiB, swizzled
  const Op* post;         // diagonal ops applied after the block
  uint32_t post_count;
  // Tensor-map load of a whole tile (blocks with no qubit below 7): the state
  // as an FP32 tensor whose dim 0 is qubits 0..6 (256 floats) and whose
  // other dims are the maximal groups of consecutive block / non-block
  // qubits above; the box is the tile (block groups at full extent). The
  // coordinate of a non-block group is the tile index bits (t >> tshift) &
  // tmaskc.
  CUtensorMap tmap;
  uint32_t trank;  // 0: per-run bulk copies instead
  uint32_t tbytes;  // bytes one box delivers (the barrier's transaction count)
  uint32_t tshift[5], tmaskc[5], tmul[5];  // coordinate d = ((t >> tshift) & tmaskc) * tmul
  const float2* coef;
  PolyTables poly;
  int* err;
  uint32_t n;
  uint32_t bq[6];
  uint64_t tmask;                       // tile qubits: block + column qubits
  uint32_t nruns, run_bytes, run_stride;  // contiguous runs of a tile; stage bytes between runs
  // Per block row j: byte offset in a stage and global offset. Kept in the
  // kernel-parameter (constant) bank so the unrolled per-element loops of the
  // converters and the epilogue read them as instruction operands.
  uint32_t rowoff[64];
  uint64_t grow[64];
  // Lane-indexed tables, copied to shared memory by the kernel.
  uint32_t coloff[128];  // byte offset of column c in a stage
  uint64_t gcol[128];    // global offset of column c
  uint64_t runoff[128];  // global offset of run r
};

// FOLD: the variant for passes whose post ops include foldable phases
// (BlockPass::fold); the plain variant keeps them out of its epilogue.
template <bool FOLD>
__global__ void __launch_bounds__(blk::THREADS, 1) block_kernel(const __grid_constant__ BlockArgs a) {
  using namespace blk;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(sm);
  uint32_t* Lcol = (uint32_t*)(sm + OFF_TAB);   // stage byte offset of column c
  uint64_t* Gcol = (uint64_t*)(Lcol + NCOL);    // global offset of column c
  uint64_t* runoff = Gcol + NCOL;               // global offset of run r
  const uint32_t bar_w = sbase + OFF_BAR;
  const uint32_t bar_sfull = bar_w + 8;         // [2] TMA -> converters: tile loaded
  const uint32_t bar_sempty = bar_sfull + 16;   // [2] converters -> TMA: stage read
  const uint32_t bar_afull = bar_sempty + 16;   // [2] converters -> MMA
  const uint32_t bar_aempty = bar_afull + 16;   // [2] MMA -> converters
  const uint32_t bar_dfull = bar_aempty + 16;   // [2] MMA -> epilogue
  const uint32_t bar_dempty = bar_dfull + 16;   // [2] epilogue -> MMA
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  __shared__ uint64_t neg_rows[MAX_POST], neg_cmask[MAX_POST];
  // Folded post phases: active for a column when (column & fold_cmask) ==
  // fold_cmask; the factor (fold_c1 when column qubit fold_col is 1, else
  // fold_c0) multiplies the rows whose block bit fold_rbit is set (all rows
  // when fold_rbit < 0).
  __shared__ uint64_t fold_cmask[MAX_POST];
  __shared__ int8_t fold_rbit[MAX_POST], fold_col[MAX_POST];
  __shared__ float2 fold_c0[MAX_POST], fold_c1[MAX_POST];
  __shared__ Op other_ops[MAX_POST];
  __shared__ int n_neg_sh, n_other_sh, n_fold_sh;
  // The non-tile qubits as runs of consecutive positions: tile index bits
  // [dep_src, dep_src + len) land on qubits [dep_dst, dep_dst + len).
  __shared__ uint32_t dep_src[16], dep_mask[16], dep_dst[16];
  __shared__ int n_dep_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t n = a.n;
  volatile int* abort_flag = &abort_sh;

  // ---- tile geometry (computed on the host) ---------------------------------
  uint64_t bmask = 0;
  for (int j = 0; j < 6; ++j) bmask |= 1ull << a.bq[j];
  const uint64_t tmask = a.tmask;
  const uint32_t nruns = a.nruns, run_bytes = a.run_bytes, run_stride = a.run_stride;
  if (tid < NCOL) {
    Lcol[tid] = a.coloff[tid];
    Gcol[tid] = a.gcol[tid];
    runoff[tid] = a.runoff[tid];
  }
  if (tid == 0) {
    mbar_init(bar_w, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_sfull + 8 * b, 1);
      mbar_init(bar_sempty + 8 * b, CONV_WARPS);
      mbar_init(bar_afull + 8 * b, CONV_WARPS);
      mbar_init(bar_aempty + 8 * b, 1);
      mbar_init(bar_dfull + 8 * b, 1);
      mbar_init(bar_dempty + 8 * b, EPI_WARPS);
    }
    fence_barrier_init();
    abort_sh = 0;
    int nd = 0;
    for (uint32_t q = 0, src = 0; q < n;) {
      if ((tmask >> q) & 1) {
        ++q;
        continue;
      }
      uint32_t len = 0;
      while (q + len < n && !((tmask >> (q + len)) & 1)) ++len;
      dep_src[nd] = src;
      dep_mask[nd] = (1u << len) - 1;  // len <= n - 13 <= 27
      dep_dst[nd] = q;
      ++nd;
      src += len;
      q += len;
    }
    n_dep_sh = nd;  // at most 14: the 13 tile qubits leave at most 14 gaps
    int nn = 0, no = 0, nf = 0;
    const uint32_t cnt = a.post_count < (uint32_t)MAX_POST ? a.post_count : (uint32_t)MAX_POST;
    for (uint32_t o = 0; o < cnt; ++o) {
      const Op op = a.post[o];
      if (op.type == OP_NEG) {
        uint64_t rows = 0;
        for (int j = 0; j < 64; ++j) {
          uint64_t gr = 0;
          for (int b = 0; b < 6; ++b)
            if ((j >> b) & 1) gr |= 1ull << a.bq[b];
          if ((gr & op.mask & bmask) == (op.mask & bmask)) rows |= 1ull << j;
        }
        neg_rows[nn] = rows;
        neg_cmask[nn] = op.mask & ~bmask;
        ++nn;
      } else if (FOLD && op.type == OP_CPHASE && __popcll(op.mask & bmask) <= 1) {
        // a phase on a corner: at most one block qubit, the rest a column condition
        const uint64_t rm = op.mask & bmask;
        int rb = -1;
        for (int b = 0; b < 6; ++b)
          if (rm == (1ull << a.bq[b])) rb = b;
        fold_cmask[nf] = op.mask & ~bmask;
        fold_rbit[nf] = (int8_t)rb;
        fold_col[nf] = -1;
        fold_c0[nf] = fold_c1[nf] = a.coef[op.coef];
        ++nf;
      } else if (FOLD && op.type == OP_DIAG && op.nq == 1 && !((bmask >> op.q[0]) & 1) && !(op.ctrl & bmask)) {
        // a one-qubit diagonal on a column qubit (controls on columns too)
        fold_cmask[nf] = op.ctrl;
        fold_rbit[nf] = -1;
        fold_col[nf] = (int8_t)op.q[0];
        fold_c0[nf] = a.coef[op.coef];
        fold_c1[nf] = a.coef[op.coef + 1];
        ++nf;
      } else {
        other_ops[no++] = op;
      }
    }
    n_neg_sh = nn;
    n_other_sh = no;
    n_fold_sh = nf;
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  const uint64_t ntiles = 1ull << (n - 13);
  const int n_dep = n_dep_sh;
  auto tile_base = [&](uint64_t t) -> uint64_t {  // deposit a tile index into the non-tile qubits
    const uint32_t tt = (uint32_t)t;              // n - 13 <= 27 bits
    uint64_t base = 0;
    for (int k = 0; k < n_dep; ++k) base |= (uint64_t)((tt >> dep_src[k]) & dep_mask[k]) << dep_dst[k];
    return base;
  };
  const uint64_t first = blockIdx.x, stride = gridDim.x;

  if (warp == TMA_WARP) {
    // ---------------- TMA: HBM -> shared-memory stages ----------------
    if (lane == 0) {
      mbar_expect_tx(bar_w, W_BYTES);
      bulk_load(sbase + OFF_W, a.image, W_BYTES, bar_w);
    }
    uint32_t i = 0;
    for (uint64_t t = first; t < ntiles; t += stride, ++i) {
      const uint32_t s = i & 1, ph = (i >> 1) & 1;
      if (!mbar_wait(bar_sempty + 8 * s, ph ^ 1, abort_flag)) {
        abort_sh = 1;
        break;
      }
      const uint32_t dst0 = sbase + OFF_S + s * STAGE_BYTES;
      if (a.trank) {
        // the whole tile as one tensor box: the copy engine's cost is per
        // copy (~100 cycles), so one box beats 64 runs of 1 KiB
        if (lane == 0) {
          mbar_expect_tx(bar_sfull + 8 * s, a.tbytes);
          int32_t crd[5];
#pragma unroll
          for (int d = 0; d < 5; ++d) crd[d] = (int32_t)(((t >> a.tshift[d]) & a.tmaskc[d]) * a.tmul[d]);
          tensor_load(dst0, &a.tmap, a.trank, crd, bar_sfull + 8 * s);
        }
        continue;
      }
      const uint64_t base = tile_base(t);
      if (lane == 0) mbar_expect_tx(bar_sfull + 8 * s, TILE_BYTES);
      __syncwarp();
      for (uint32_t r = lane; r < nruns; r += 32)
        bulk_load(dst0 + r * run_stride, a.amps + (base | runoff[r]), run_bytes, bar_sfull + 8 * s);
    }
  } else if (warp >= CONV_WARP0 && warp < CONV_WARP0 + CONV_WARPS) {
    // ---------------- converters: stage -> BF16 hi/lo -> TMEM A operand ----------------
    const int q = warp & 3;  // TMEM lane quarter
    const int col = 32 * q + lane;
    const uint32_t lc = Lcol[col];
    // With qubit 0 in the block, block rows 2p and 2p+1 sit 8 bytes apart in
    // the stage and every row pair starts on a 16-byte boundary (all other
    // stage strides are multiples of 16).
    const bool row_pairs = a.bq[0] == 0;
    uint32_t i = 0;
    for (uint64_t t = first; t < ntiles; t += stride, ++i) {
      const uint32_t s = i & 1, ph = (i >> 1) & 1;
      if (!mbar_wait(bar_sfull + 8 * s, ph, abort_flag) || !mbar_wait(bar_aempty + 8 * s, ph ^ 1, abort_flag)) {
        abort_sh = 1;
        break;
      }
      tc_fence_after();
      const uint8_t* stg = sm + OFF_S + s * STAGE_BYTES + lc;  // this thread's column
      const uint32_t ta = tmem + TM_A + 128 * s + ((uint32_t)(32 * q) << 16);  // this warp's lanes
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {  // block rows 32h .. 32h+31
        uint32_t hr[16], hi[16], lr[16], li[16];
#pragma unroll
        for (int p = 0; p < 16; ++p) {
          const uint32_t r0 = h ? a.rowoff[32 + 2 * p] : a.rowoff[2 * p];
          const uint32_t r1 = h ? a.rowoff[33 + 2 * p] : a.rowoff[2 * p + 1];
          float2 x0, x1;
          if (row_pairs) {  // rows 2p, 2p+1 adjacent: one 16-byte load
            const float4 v = *(const float4*)(stg + r0);
            x0 = make_float2(v.x, v.y);
            x1 = make_float2(v.z, v.w);
          } else {
            x0 = *(const float2*)(stg + r0);
            x1 = *(const float2*)(stg + r1);
          }
          split_pair(x0.x, x1.x, hr[p], lr[p]);
          split_pair(x0.y, x1.y, hi[p], li[p]);
        }
        // A row layout: K = [Re x_0..63 | Im x_0..63], two BF16 per 32-bit column
        tmem_st16(ta + 16 * h, hr);            // hi, Re part
        tmem_st16(ta + 32 + 16 * h, hi);       // hi, Im part
        tmem_st16(ta + 64 + 16 * h, lr);       // lo, Re part
        tmem_st16(ta + 64 + 32 + 16 * h, li);  // lo, Im part
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(bar_sempty + 8 * s);  // this warp is done reading the stage
      tc_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar_afull + 8 * s);
    }
  } else if (warp == MMA_WARP) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      if (!mbar_wait(bar_w, 0, abort_flag)) abort_sh = 1;
      uint32_t i = 0;
      for (uint64_t t = first; t < ntiles && !*abort_flag; t += stride, ++i) {
        const uint32_t b = i & 1, ph = (i >> 1) & 1;
        if (!mbar_wait(bar_afull + 8 * b, ph, abort_flag) || !mbar_wait(bar_dempty + 8 * b, ph ^ 1, abort_flag)) {
          abort_sh = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + TM_D + 128 * b;
        const uint32_t ah = tmem + TM_A + 128 * b, al = ah + 64;
        const uint32_t at[3] = {ah, al, ah};
        const uint32_t wb[3] = {sbase + OFF_W, sbase + OFF_W, sbase + OFF_W + W_BYTES / 2};
#pragma unroll
        for (int term = 0; term < 3; ++term)
#pragma unroll
          for (int ks = 0; ks < 8; ++ks) {
            const uint32_t koff = (ks >> 2) * (128 * 128) + (ks & 3) * 32;
            tc_mma_ts(d, at[term] + 8 * ks, sw128_desc(wb[term] + koff), IDESC, (term | ks) ? 1u : 0u);
          }
        tc_commit(bar_aempty + 8 * b);  // A buffer free once these MMAs complete
        tc_commit(bar_dfull + 8 * b);   // accumulator ready
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: TMEM -> registers -> HBM ----------------
    // A block on qubit 0 keeps row pairs (2p, 2p+1) adjacent in HBM: each
    // thread then writes them as one 16-byte store.
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int h = (warp - EPI_WARP0) >> 2;  // block rows 32h .. 32h+31
    const int col = 32 * q + lane;
    const bool pairs = a.bq[0] == 0;
    // With qubits 0, 1, 2 as block bits 0..2, rows 8k .. 8k+7 of a column are
    // 64 contiguous bytes in HBM: those tiles are written through a small
    // per-warp shared-memory transpose (32 columns x 8 rows).
    const bool octets = pairs && a.bq[1] == 1 && a.bq[2] == 2;
    float4* ep = (float4*)(sm + OFF_EPI + EPI_STAGE_BYTES * (warp - EPI_WARP0));
    const int n_neg = n_neg_sh, n_other = n_other_sh, n_fold = n_fold_sh;
    uint32_t i = 0;
    for (uint64_t t = first; t < ntiles; t += stride, ++i) {
      const uint32_t b = i & 1, ph = (i >> 1) & 1;
      const uint64_t tb = tile_base(t);
      const uint64_t gc = tb | Gcol[col];
      uint64_t neg = 0;
      for (int o = 0; o < n_neg; ++o)
        if ((gc & neg_cmask[o]) == neg_cmask[o]) neg ^= neg_rows[o];
      // folded phases of this column: a factor for every row (fb) and one per
      // block-row bit (fr[0..5])
      float2 fb = make_float2(1.f, 0.f), fr[6];
#pragma unroll
      for (int r = 0; r < 6; ++r) fr[r] = make_float2(1.f, 0.f);
      for (int o = 0; FOLD && o < n_fold; ++o) {
        if ((gc & fold_cmask[o]) != fold_cmask[o]) continue;
        const int cq = fold_col[o];
        const float2 c = (cq >= 0 && ((gc >> cq) & 1)) ? fold_c1[o] : fold_c0[o];
        const int rb = fold_rbit[o];
        if (rb < 0) fb = cmul<float>(fb, c);
#pragma unroll
        for (int r = 0; r < 6; ++r)
          if (rb == r) fr[r] = cmul<float>(fr[r], c);
      }
      if (!mbar_wait(bar_dfull + 8 * b, ph, abort_flag)) {
        abort_sh = 1;
        break;
      }
      tc_fence_after();
      const uint32_t tl = tmem + TM_D + 128 * b + ((uint32_t)(32 * q) << 16);
      {
        float re[32], im[32];
        tmem_ld32(tl + 32 * h, re);
        tmem_ld32(tl + 64 + 32 * h, im);
        tc_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_dempty + 8 * b);  // accumulator read: the MMA may reuse it
        const uint32_t negh = (uint32_t)(neg >> (32 * h));
        float2* pc = a.amps + gc;
        // separate copies of the row loop, so that passes without folded
        // phases or general post ops keep the plain one
        auto store_rows = [&](auto fold_tag, auto other_tag, auto octet_tag) {
          constexpr bool WITH_FOLD = decltype(fold_tag)::value;
          constexpr bool WITH_OTHER = decltype(other_tag)::value;
          constexpr bool OCTETS = decltype(octet_tag)::value;
          const float2 fh = h ? cmul<float>(fb, fr[5]) : fb;  // row bit 5 is this warp's half
#pragma unroll
          for (int jj = 0; jj < 32; jj += 2) {
            float2 y0 = make_float2(re[jj], im[jj]), y1 = make_float2(re[jj + 1], im[jj + 1]);
            if ((negh >> jj) & 1) y0 = make_float2(-y0.x, -y0.y);
            if ((negh >> (jj + 1)) & 1) y1 = make_float2(-y1.x, -y1.y);
            if constexpr (WITH_FOLD) {
              float2 f0 = fh;
#pragma unroll
              for (int r = 1; r < 5; ++r)
                if ((jj >> r) & 1) f0 = cmul<float>(f0, fr[r]);
              y0 = cmul<float>(f0, y0);
              y1 = cmul<float>(cmul<float>(f0, fr[0]), y1);  // row jj + 1 adds bit 0
            }
            const uint64_t g0 = h ? a.grow[32 + jj] : a.grow[jj];
            const uint64_t g1 = h ? a.grow[33 + jj] : a.grow[jj + 1];
            if constexpr (WITH_OTHER) {
              // general post ops (rare): stage this thread's 8-row chunk in
              // its own slots of the warp's buffer, then apply them in a
              // rolled loop and store from there
              float2* eo = (float2*)ep;  // [row in chunk][lane]
              eo[(jj & 7) * 32 + lane] = y0;
              eo[((jj & 7) + 1) * 32 + lane] = y1;
              if ((jj & 7) == 6) {
                const int j0 = 32 * h + (jj & ~7);
#pragma unroll 1
                for (int r = 0; r < 8; ++r) {
                  float2 y = eo[r * 32 + lane];
                  const uint64_t g = a.grow[j0 + r];
                  for (int o = 0; o < n_other; ++o) y = apply_diag_op<float>(other_ops[o], y, gc | g, a.coef, a.poly);
                  __stcs(pc + g, y);
                }
              }
            } else if constexpr (OCTETS) {
              // stage the row pair; after every 8 rows the warp writes them
              // out column by column, 64 contiguous bytes per column (8 lines
              // per store instruction instead of 32)
              ep[4 * lane + (((jj & 7) >> 1) ^ ((lane >> 1) & 3))] = make_float4(y0.x, y0.y, y1.x, y1.y);
              if ((jj & 7) == 6) {
                __syncwarp();
                const uint64_t gr = h ? a.grow[32 + (jj & ~7)] : a.grow[jj & ~7];
                const int qd = lane & 3;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                  const int c = 8 * m + (lane >> 2);
                  const float4 v = ep[4 * c + (qd ^ ((c >> 1) & 3))];
                  __stcs((float4*)(a.amps + ((tb | Gcol[32 * q + c]) + gr + 2 * qd)), v);
                }
                __syncwarp();
              }
            } else if (pairs) {
              __stcs((float4*)(pc + g0), make_float4(y0.x, y0.y, y1.x, y1.y));
            } else {
              __stcs(pc + g0, y0);
              __stcs(pc + g1, y1);
            }
          }
        };
        if (n_other)
          store_rows(std::integral_constant<bool, FOLD>{}, std::true_type{}, std::false_type{});
        else if (octets)
          store_rows(std::integral_constant<bool, FOLD>{}, std::false_type{}, std::true_type{});
        else
          store_rows(std::integral_constant<bool, FOLD>{}, std::false_type{}, std::false_type{});
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (abort_sh && tid == 0) atomicExch(a.err, ALEPH_B200_DEVICE_FAILURE);
  if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
}

namespace {

// Bank-conflict degree of one warp's 8-byte shared-memory accesses at byte
// offsets off[0..32): the most distinct 4-byte words any of the 32 banks
// serves (2 is the minimum: 256 bytes take two 128-byte wavefronts).
int conflict_degree(const uint32_t* off) {
  int worst = 0;
  for (uint32_t bank = 0; bank < 32; ++bank) {
    uint32_t words[64];
    int nw = 0;
    for (int t = 0; t < 32; ++t)
      for (uint32_t h = 0; h < 2; ++h) {
        const uint32_t w = off[t] / 4 + h;
        if (w % 32 != bank) continue;
        bool seen = false;
        for (int k = 0; k < nw; ++k) seen = seen || words[k] == w;
        if (!seen) words[nw++] = w;
      }
    worst = nw > worst ? nw : worst;
  }
  return worst;
}

// Tile geometry of a block pass. The tile qubits are the 6 block qubits plus
// 7 column qubits; a tile is 2^(13-c) contiguous runs of 2^c amplitudes
// (qubits 0..c-1 all in the tile), kept in a stage back to back, each run
// followed by `pad` bytes. Column candidates: the 7 lowest non-block qubits,
// and, for a block with a qubit below 7 that ends at or below qubit 12, the
// non-block qubits under the block plus the ones above a one-qubit gap after
// it (so that those columns index runs, which the pad skews across banks).
// The candidate and pad with the fewest bank conflicts for the 32 columns of
// a warp win (ties: the first, natural and unpadded).
void set_tile_geometry(uint32_t n, const uint32_t* bq, BlockArgs* a) {
  using namespace blk;
  uint64_t bmask = 0;
  uint32_t bmax = 0;
  for (int j = 0; j < 6; ++j) {
    bmask |= 1ull << bq[j];
    bmax = bq[j] > bmax ? bq[j] : bmax;
  }
  uint32_t cand[2][7];
  int ncand = 0;
  {
    int k = 0;
    for (uint32_t q = 0; q < n && k < 7; ++q)
      if (!((bmask >> q) & 1)) cand[ncand][k++] = q;
    ++ncand;
  }
  if ((bmask & 0x7F) && bmax <= 12) {
    int k = 0;
    for (uint32_t q = 0; q < bmax; ++q)
      if (!((bmask >> q) & 1)) cand[ncand][k++] = q;
    for (uint32_t q = bmax + 2; q < n && k < 7; ++q) cand[ncand][k++] = q;
    if (k == 7) ++ncand;
  }
  int best_deg = 1 << 30, best_c = 0;
  uint32_t best_pad = 0;
  for (int ci = 0; ci < ncand; ++ci) {
    uint64_t tmask = bmask;
    for (int k = 0; k < 7; ++k) tmask |= 1ull << cand[ci][k];
    uint32_t c = 0;
    while (c < 13 && ((tmask >> c) & 1)) ++c;
    const uint32_t nruns = 1u << (13 - c), run_bytes = 8u << c;
    for (uint32_t pad : {0u, 16u, 32u, 64u, 128u, 256u, 512u}) {
      if (nruns * pad > (uint32_t)MAX_PAD_BYTES) break;
      uint32_t off[32];
      for (int t = 0; t < 32; ++t) {
        off[t] = 0;
        for (int k = 0; k < 5; ++k) {
          if (!((t >> k) & 1)) continue;
          const uint32_t pos = (uint32_t)__builtin_popcountll(tmask & ((1ull << cand[ci][k]) - 1));
          off[t] += pos < c ? 8u << pos : (run_bytes + pad) << (pos - c);
        }
      }
      const int deg = conflict_degree(off);
      if (deg < best_deg) {
        best_deg = deg;
        best_c = ci;
        best_pad = pad;
      }
    }
  }
  const uint32_t* cols = cand[best_c];
  uint64_t tmask = bmask;
  for (int k = 0; k < 7; ++k) tmask |= 1ull << cols[k];
  uint32_t c = 0;
  while (c < 13 && ((tmask >> c) & 1)) ++c;
  a->tmask = tmask;
  a->nruns = 1u << (13 - c);
  a->run_bytes = 8u << c;
  a->run_stride = a->run_bytes + best_pad;
  auto stride = [&](uint32_t q) -> uint32_t {  // stage byte stride of tile qubit q
    const uint32_t pos = (uint32_t)__builtin_popcountll(tmask & ((1ull << q) - 1));
    return pos < c ? 8u << pos : a->run_stride << (pos - c);
  };
  for (uint32_t j = 0; j < 64; ++j) {
    uint32_t ro = 0;
    uint64_t gr = 0;
    for (int b = 0; b < 6; ++b)
      if ((j >> b) & 1) {
        ro += stride(bq[b]);
        gr |= 1ull << bq[b];
      }
    a->rowoff[j] = ro;
    a->grow[j] = gr;
  }
  for (uint32_t col = 0; col < (uint32_t)NCOL; ++col) {
    uint32_t co = 0;
    uint64_t gc = 0;
    for (int k = 0; k < 7; ++k)
      if ((col >> k) & 1) {
        co += stride(cols[k]);
        gc |= 1ull << cols[k];
      }
    a->coloff[col] = co;
    a->gcol[col] = gc;
  }
  for (uint32_t r = 0; r < (uint32_t)MAX_RUNS; ++r) {  // run r: its bits -> the tile qubits from c up
    uint64_t off = 0;
    if (r < a->nruns) {
      uint32_t bit = 0;
      for (uint32_t q = c; q < n; ++q)
        if ((tmask >> q) & 1) {
          if ((r >> bit) & 1) off |= 1ull << q;
          ++bit;
        }
    }
    a->runoff[r] = off;
  }
}

// The tensor map of a tile box (BlockArgs::tmap), for two geometries:
//  * a block with no qubit below 7, whose tile is 64 unpadded runs of 1 KiB:
//    dim 0 is qubits 0..6 (256 floats, the box's full width), then the
//    maximal groups of consecutive block / non-block qubits;
//  * the block on qubits 0..5 with its columns on qubits 7..13 (above the
//    gap at qubit 6), whose tile is 128 runs of 512 B each followed by a
//    16-byte pad: dim 0 is qubits 0..6 and the box takes 132 floats of it
//    (a column's 64 amplitudes plus 16 bytes that land in the pad; the
//    tile's qubit-6 bit is the x offset 0 or 128 floats), dim 1 the 128
//    columns, dim 2 the qubits from 14 up.
// Leaves trank = 0 (per-run bulk copies) for any other geometry, for more
// than 5 dimensions, or when the driver's encoder is unavailable or refuses
// the map.
void set_tensor_map(uint32_t n, void* amps, BlockArgs* a) {
  using namespace blk;
  a->trank = 0;
  uint64_t bmask = 0;
  for (int j = 0; j < 6; ++j) bmask |= 1ull << a->bq[j];
  const bool high = !(bmask & 0x7F) && a->nruns == 64 && a->run_bytes == 1024 && a->run_stride == 1024;
  const bool low = bmask == 0x3F && a->tmask == 0x3FBFull && a->nruns == 128 && a->run_bytes == 512 &&
                   a->run_stride == 528 && n >= 14;
  if (!high && !low) return;
  typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = (EncodeFn)fn;
  }
  if (!encode) return;
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < 5; ++d) {
    a->tshift[d] = a->tmaskc[d] = 0;
    a->tmul[d] = 1;
  }
  gdim[0] = 256;  // qubits 0..6: 128 complex = 256 floats, 1 KiB
  if (low) {
    box[0] = 132;  // 512 B of a column + 16 B into the pad
    a->tmaskc[0] = 1;  // tile bit 0 is qubit 6: x = 0 or 128 floats
    a->tmul[0] = 128;
    gdim[1] = 128;  // columns: qubits 7..13
    gstride[0] = 8ull << 7;
    box[1] = 128;
    gdim[2] = 1ull << (n - 14);  // qubits 14..n-1: tile bits 1..
    gstride[1] = 8ull << 14;
    box[2] = 1;
    a->tshift[2] = 1;
    a->tmaskc[2] = (uint32_t)((1ull << (n - 14)) - 1);
    const CUresult r = encode(&a->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, amps, gdim, gstride, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS) {
      a->trank = 3;
      a->tbytes = 132 * 128 * 4;
    }
    return;
  }
  box[0] = 256;
  uint32_t rank = 1, tbit = 0;
  for (uint32_t q = 7; q < n;) {
    const bool blockq = (bmask >> q) & 1;
    uint32_t len = 0;
    while (q + len < n && (((bmask >> (q + len)) & 1) != 0) == blockq) ++len;
    if (rank == 5) return;
    gdim[rank] = 1ull << len;
    gstride[rank - 1] = 8ull << q;
    box[rank] = blockq ? (1u << len) : 1u;
    a->tshift[rank] = blockq ? 0 : tbit;
    a->tmaskc[rank] = blockq ? 0 : (uint32_t)((1ull << len) - 1);
    if (!blockq) tbit += len;
    ++rank;
    q += len;
  }
  if (rank < 2) return;
  const CUresult r = encode(&a->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, amps, gdim, gstride, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS) {
    a->trank = rank;
    a->tbytes = TILE_BYTES;
  }
}

}  // namespace

cudaError_t launch_block_pass(void* amps, const BlockPass& p, const uint8_t* images, const Op* ops, const void* coef,
                              PolyTables poly, int* dev_error, int sm_count, cudaStream_t s) {
  if (p.n < 13) return cudaErrorInvalidValue;
  BlockArgs a;
  a.amps = (float2*)amps;
  a.image = images + p.mat;
  a.post = ops + p.post_begin;
  a.post_count = p.post_count;
  a.coef = (const float2*)coef;
  a.poly = poly;
  a.err = dev_error;
  a.n = p.n;
  for (int j = 0; j < 6; ++j) a.bq[j] = p.bq[j];
  set_tile_geometry(p.n, p.bq, &a);
  set_tensor_map(p.n, amps, &a);
  static uint64_t attr_devices = 0;  // devices on which the shared-memory opt-in is done
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 64 || !((attr_devices >> dev) & 1)) {
    e = cudaFuncSetAttribute(block_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, blk::SMEM_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(block_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, blk::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_devices |= 1ull << dev;
  }
  const uint64_t ntiles = 1ull << (p.n - 13);
  const unsigned grid = (unsigned)(ntiles < (uint64_t)sm_count ? ntiles : (uint64_t)sm_count);
  if (p.fold)
    block_kernel<true><<<grid, blk::THREADS, blk::SMEM_BYTES, s>>>(a);
  else
    block_kernel<false><<<grid, blk::THREADS, blk::SMEM_BYTES, s>>>(a);
  return cudaGetLastError();
}

// Host helper: lay out a 128x128 real matrix (row-major doubles, W[r][k]) as
// the split BF16 hi / lo K-major SW128 images the kernel loads (64 KiB).
void build_block_image(const double* W, uint8_t* out) {
  uint16_t* hi = (uint16_t*)out;
  uint16_t* lo = (uint16_t*)(out + blk::W_BYTES / 2);
  auto to_bf16 = [](float f) -> uint16_t {  // round to nearest even
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
  };
  auto from_bf16 = [](uint16_t b) -> float {
    uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  for (uint32_t m = 0; m < 128; ++m)
    for (uint32_t k = 0; k < 128; ++k) {
      const float w = (float)W[m * 128 + k];
      const uint16_t h = to_bf16(w);
      const uint16_t l = to_bf16(w - from_bf16(h));
      const uint32_t off = blk::sw128_off(m, k, 128) / 2;
      hi[off] = h;
      lo[off] = l;
    }
}

}  // namespace ab
