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
// The state columns form the MMA's M dimension (TMEM lanes) and the 128 output
// rows its N dimension, so in the epilogue each thread owns one column with
// both the real and imaginary part of each of its outputs: complex results
// (and the diagonal ops that follow the block) stay in registers and go to
// shared memory as 8-byte stores across consecutive columns.
//
// Per CTA (persistent, one per SM, 8 warps):
//   * W_hi / W_lo arrive once as prebuilt BF16 images in the UMMA canonical
//     K-major 128-byte-swizzled layout (cp.async.bulk, 64 KiB, the B operand);
//   * each tile (64 block rows x 128 columns, 64 KiB FP32) is fetched by plain
//     (non-multicast) cp.async.bulk copies of its contiguous runs, completion
//     tracked by an mbarrier transaction count; the next tile's fetch is issued
//     as soon as the current one has been split, overlapping the MMAs, the
//     epilogue and the store;
//   * all threads split the tile into X_hi / X_lo (the A operand, same
//     canonical layout), one thread issues 3 x 8 tcgen05.mma (M=128, N=128,
//     K=16, kind::f16, BF16 inputs, FP32 accumulate) and commits to an
//     mbarrier;
//   * the epilogue reads the accumulator with tcgen05.ld (32x32b), applies
//     the diagonal ops after the block, writes the FP32 tile into the operand
//     buffer (free once the MMAs completed) and stores it with cp.async.bulk.
// Every wait is bounded; on expiry the CTA records an error code, drains its
// own bulk copies, frees its TMEM and returns.

#include <cstdint>
#include <cstring>

#include <cuda_bf16.h>

#include "common.cuh"

namespace ab {

namespace blk {

constexpr int THREADS = 256;
constexpr int NCOL = 128;                     // columns per tile (MMA M)
constexpr int TILE_AMPS = 64 * NCOL;          // 8192 complex
constexpr int TILE_BYTES = TILE_AMPS * 8;     // 64 KiB FP32 complex
constexpr int W_BYTES = 2 * 128 * 128 * 2;    // hi + lo images, 64 KiB
constexpr int X_PART = NCOL * 128 * 2;        // one BF16 operand part, 32 KiB
constexpr uint32_t TMEM_COLS = 128;
constexpr long long SPIN_LIMIT = 1ll << 28;   // bounded mbarrier waits

// shared-memory map (offsets from a 1024-byte aligned base)
constexpr int OFF_W = 0;                                  // B operand: W_hi | W_lo
constexpr int OFF_X = OFF_W + W_BYTES;                    // A operand: X_hi | X_lo, then the FP32 output tile
constexpr int OFF_S = OFF_X + 2 * X_PART;                 // input tile
constexpr int OFF_TAB = OFF_S + TILE_BYTES;               // index tables
constexpr int TAB_BYTES = 64 * 4 + NCOL * 4 + 64 * 8 + 64 * 8 + NCOL * 8;
constexpr int OFF_BAR = OFF_TAB + TAB_BYTES;              // mbarriers
constexpr int SMEM_BYTES = OFF_BAR + 64 + 1024;           // + alignment slack
static_assert(2 * X_PART == TILE_BYTES, "the output tile reuses the operand buffer");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
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
// Bounded wait: false on expiry.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < SPIN_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

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
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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

__device__ __forceinline__ uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_val(uint32_t b) { return __uint_as_float(b << 16); }

}  // namespace blk

// Kernel parameters beyond BlockPass.
struct BlockArgs {
  float2* amps;
  const uint8_t* image;   // W_hi | W_lo, 64 KiB, swizzled
  const Op* post;         // diagonal ops applied after the block
  uint32_t post_count;
  const float2* coef;
  PolyTables poly;
  int* err;
  uint32_t n;
  uint32_t bq[6];
};

__global__ void __launch_bounds__(blk::THREADS, 1) block_kernel(const BlockArgs a) {
  using namespace blk;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(sm);
  uint32_t* Lrow = (uint32_t*)(sm + OFF_TAB);  // local index of block row j
  uint32_t* Lcol = Lrow + 64;                  // local index of column c
  uint64_t* runoff = (uint64_t*)(Lcol + NCOL); // global offset of run r
  uint64_t* Grow = runoff + 64;                // global offset of block row j
  uint64_t* Gcol = Grow + 64;                  // global offset of column c
  const uint32_t bar_full = sbase + OFF_BAR;
  const uint32_t bar_w = bar_full + 8;
  const uint32_t bar_mma = bar_w + 8;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  __shared__ uint64_t tile_base_sh;
  // post-block diagonal ops: sign flips (CZ-like) as (row mask over j, column-side mask) pairs;
  // everything else as cached Op records applied per element
  constexpr int MAX_POST = 48;
  __shared__ uint64_t neg_rows[MAX_POST], neg_cmask[MAX_POST];
  __shared__ Op other_ops[MAX_POST];
  __shared__ int n_neg_sh, n_other_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t n = a.n;

  // ---- tile geometry -------------------------------------------------------
  // Tile qubit set T = block qubits + the 7 lowest other qubits (the column
  // bits). T contains all qubits 0..c-1 (one contiguous run of 2^c
  // amplitudes) plus the block qubits above them; local index bits follow T
  // in ascending order.
  uint64_t bmask = 0;
  for (int j = 0; j < 6; ++j) bmask |= 1ull << a.bq[j];
  uint32_t cols[7];
  {
    int k = 0;
    for (uint32_t q = 0; q < n && k < 7; ++q)
      if (!((bmask >> q) & 1)) cols[k++] = q;
  }
  uint64_t tmask = bmask;
  for (int k = 0; k < 7; ++k) tmask |= 1ull << cols[k];
  uint32_t c = 0;
  while (c < 13 && ((tmask >> c) & 1)) ++c;  // contiguous run: qubits 0..c-1
  const uint32_t nruns = 1u << (13 - c), run_bytes = (1u << c) * 8;
  auto local_pos = [&](uint32_t q) -> uint32_t { return (uint32_t)__popcll(tmask & ((1ull << q) - 1)); };
  if (tid < NCOL) {
    uint32_t lc = 0;
    uint64_t gc = 0;
    for (int k = 0; k < 7; ++k)
      if ((tid >> k) & 1) {
        lc |= 1u << local_pos(cols[k]);
        gc |= 1ull << cols[k];
      }
    Lcol[tid] = lc;
    Gcol[tid] = gc;
  }
  if (tid < 64) {
    uint32_t lr = 0;
    uint64_t gr = 0;
    for (int j = 0; j < 6; ++j)
      if ((tid >> j) & 1) {
        lr |= 1u << local_pos(a.bq[j]);
        gr |= 1ull << a.bq[j];
      }
    Lrow[tid] = lr;
    Grow[tid] = gr;
    // run r: local bits c..12 -> the T qubits above c-1
    uint64_t off = 0;
    if ((uint32_t)tid < nruns) {
      uint32_t bit = 0;
      for (uint32_t q = c; q < n; ++q)
        if ((tmask >> q) & 1) {
          if ((tid >> bit) & 1) off |= 1ull << q;
          ++bit;
        }
    }
    runoff[tid] = off;
  }
  if (tid == 0) {
    mbar_init(bar_full, 1);
    mbar_init(bar_w, 1);
    mbar_init(bar_mma, 1);
    fence_barrier_init();
    abort_sh = 0;
    int nn = 0, no = 0;
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
      } else {
        other_ops[no++] = op;
      }
    }
    n_neg_sh = nn;
    n_other_sh = no;
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
    tmem_relinquish();
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  const uint64_t ntiles = 1ull << (n - 13);
  // deposit a tile index into the non-T qubits
  auto tile_base = [&](uint64_t t) -> uint64_t {
    uint64_t base = 0;
    for (uint32_t q = 0; t != 0 && q < n; ++q) {
      if ((tmask >> q) & 1) continue;
      base |= (t & 1) << q;
      t >>= 1;
    }
    return base;
  };
  // The runs of a tile are fetched by the 32 lanes of warp 0 together (lane 0
  // posts the byte count first) and stored back by the lanes of warp 1, so no
  // single thread serialises up to 64 bulk copies per direction.
  auto issue_tile = [&](uint64_t t) {  // all lanes of warp 0
    const uint64_t base = tile_base(t);
    if (lane == 0) mbar_expect_tx(bar_full, TILE_BYTES);
    __syncwarp();
    for (uint32_t r = lane; r < nruns; r += 32)
      bulk_load(sbase + OFF_S + r * run_bytes, a.amps + (base | runoff[r]), run_bytes, bar_full);
  };

  const uint64_t first = blockIdx.x, stride = gridDim.x;
  if (warp == 0) {
    if (lane == 0) {
      mbar_expect_tx(bar_w, W_BYTES);
      bulk_load(sbase + OFF_W, a.image, W_BYTES, bar_w);
    }
    if (first < ntiles) issue_tile(first);
  }
  if (!mbar_wait(bar_w, 0)) abort_sh = 1;
  __syncthreads();

  const float2* stg = (const float2*)(sm + OFF_S);
  float2* out = (float2*)(sm + OFF_X);
  uint32_t it = 0;
  for (uint64_t t = first; t < ntiles && !abort_sh; t += stride, ++it) {
    if (!mbar_wait(bar_full, it & 1)) abort_sh = 1;
    if (warp == 1) bulk_wait_read0();  // each storing lane: its copies have read the operand buffer
    if (tid == 0) tile_base_sh = tile_base(t);
    __syncthreads();
    if (abort_sh) break;

    // ---- split the FP32 tile into BF16 hi/lo operands (A: 128 columns x K=128) ----
    // item = (column col, 8-row group g): 8 complex -> 4 x 16-byte chunks
    for (int item = tid; item < NCOL * 8; item += THREADS) {
      const int col = item & (NCOL - 1), g = item >> 7;
      const uint32_t lc = Lcol[col];
      uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        const float2 x0 = stg[Lrow[8 * g + e] | lc];
        const float2 x1 = stg[Lrow[8 * g + e + 1] | lc];
        const uint32_t h0 = bf16_bits(x0.x), h1 = bf16_bits(x1.x);
        const uint32_t l0 = bf16_bits(x0.x - bf16_val(h0)), l1 = bf16_bits(x1.x - bf16_val(h1));
        const uint32_t j0 = bf16_bits(x0.y), j1 = bf16_bits(x1.y);
        const uint32_t m0 = bf16_bits(x0.y - bf16_val(j0)), m1 = bf16_bits(x1.y - bf16_val(j1));
        rh[e >> 1] = h0 | (h1 << 16);
        rl[e >> 1] = l0 | (l1 << 16);
        ih[e >> 1] = j0 | (j1 << 16);
        il[e >> 1] = m0 | (m1 << 16);
      }
      const uint32_t ore = sw128_off(col, 8 * g, NCOL), oim = sw128_off(col, 64 + 8 * g, NCOL);
      *(uint4*)(sm + OFF_X + ore) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
      *(uint4*)(sm + OFF_X + X_PART + ore) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
      *(uint4*)(sm + OFF_X + oim) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
      *(uint4*)(sm + OFF_X + X_PART + oim) = make_uint4(il[0], il[1], il[2], il[3]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0) {
      // the input buffer is free: fetch the next tile while this one computes
      const uint64_t nt = t + stride;
      if (nt < ntiles) issue_tile(nt);
    }
    if (tid == 32) {
      // ---- 3 x 8 tensor-core MMAs: D = Xh Wh + Xl Wh + Xh Wl ----
      const uint32_t xa[3] = {sbase + OFF_X, sbase + OFF_X + X_PART, sbase + OFF_X};
      const uint32_t wb[3] = {sbase + OFF_W, sbase + OFF_W, sbase + OFF_W + W_BYTES / 2};
#pragma unroll
      for (int term = 0; term < 3; ++term)
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          const uint32_t koff = (ks >> 2) * (128 * 128) + (ks & 3) * 32;  // both operands have 128 rows
          tc_mma(tmem, sw128_desc(xa[term] + koff), sw128_desc(wb[term] + koff), IDESC, (term | ks) ? 1u : 0u);
        }
      tc_commit(bar_mma);
    }
    if (!mbar_wait(bar_mma, it & 1)) abort_sh = 1;
    tc_fence_after();

    // ---- epilogue: TMEM -> registers -> post-block diagonal ops -> FP32 tile ----
    {
      const int q = warp & 3, h = warp >> 2;  // columns 32q + lane; block rows 32h..32h+31
      const int col = 32 * q + lane;
      float re[32], im[32];
      const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
      tmem_ld32(tl + 32 * h, re);
      tmem_ld32(tl + 64 + 32 * h, im);
      tc_wait_ld();
      const uint32_t lc = Lcol[col];
      const uint64_t gc = tile_base_sh | Gcol[col];
      // sign flips of the CZ-like post ops for this column, as a mask over rows j
      uint64_t neg = 0;
      for (int o = 0; o < n_neg_sh; ++o)
        if ((gc & neg_cmask[o]) == neg_cmask[o]) neg ^= neg_rows[o];
      const uint32_t negh = (uint32_t)(neg >> (32 * h));
      const int n_other = n_other_sh;
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) {
        float2 y = make_float2(re[jj], im[jj]);
        if ((negh >> jj) & 1) y = make_float2(-y.x, -y.y);
        if (n_other) {
          const uint64_t g = gc | Grow[32 * h + jj];
          for (int o = 0; o < n_other; ++o) y = apply_diag_op<float>(other_ops[o], y, g, a.coef, a.poly);
        }
        out[Lrow[32 * h + jj] | lc] = y;
      }
    }
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
    if (warp == 1) {
      const uint64_t base = tile_base_sh;
      for (uint32_t r = lane; r < nruns; r += 32)
        bulk_store(a.amps + (base | runoff[r]), sbase + OFF_X + r * run_bytes, run_bytes);
      bulk_commit();
    }
  }
  // drain: bulk copies must finish with shared memory before exit
  if (warp == 1) bulk_wait0();
  if (abort_sh) {
    // a fetch may still be in flight after an expired wait: give it a bounded chance to land
    if (tid == 0) mbar_wait(bar_full, it & 1);
    if (tid == 0) atomicExch(a.err, ALEPH_B200_DEVICE_FAILURE);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
}

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
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, blk::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const uint64_t ntiles = 1ull << (p.n - 13);
  const unsigned grid = (unsigned)(ntiles < (uint64_t)sm_count ? ntiles : (uint64_t)sm_count);
  block_kernel<<<grid, blk::THREADS, blk::SMEM_BYTES, s>>>(a);
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
