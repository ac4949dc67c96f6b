// kernels_misc.cu — shared-memory whole-state pass (n <= 12), dense k-qubit
// UnitaryKq pass, state initialisation, precision conversion and the in-place
// qubit permutation (relabelled SWAPs, unpermute_state).
//
// Semantics follow the reference kernels: pair/quartet butterflies
// (crates/aleph-sv/src/kernels/aos.rs:192-223, :1335-1394), MSB-first operand
// order (crates/aleph-sv/src/kernels/unitary_kq.rs:66-96), controls as an AND
// mask over the basis index (aos.rs:198-205).

#include <cstdio>
#include <cstring>

#include "common.cuh"

namespace ab {

// ---- whole state in shared memory (n <= 12) ---------------------------------
template <typename Real>
__device__ void smem_apply_op(V2<Real>* sm, uint32_t n, const Op& op, const V2<Real>* coef, const PolyTables& poly) {
  const uint64_t len = 1ull << n;
  const V2<Real>* m = coef + op.coef;
  if (is_diag_type(op.type)) {
    for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) sm[i] = apply_diag_op<Real>(op, sm[i], i, coef, poly);
    return;
  }
  const int k = op.type == OP_2Q ? 2 : (op.type == OP_KQ ? op.nq : 1);
  uint32_t sorted[6];
  for (int i = 0; i < k; ++i) sorted[i] = op.q[i];
  for (int i = 1; i < k; ++i)
    for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; --j) {
      uint32_t t = sorted[j];
      sorted[j] = sorted[j - 1];
      sorted[j - 1] = t;
    }
  const uint32_t dim = 1u << k;
  const uint64_t groups = len >> k;
  for (uint64_t gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    uint64_t base = gi;
    for (int i = 0; i < k; ++i) base = insert_zero(base, sorted[i]);
    if ((base & op.ctrl) != op.ctrl) continue;
    // offsets[c]: matrix bit p <-> qubit q[k-1-p]
    auto off = [&](uint32_t c) {
      uint64_t o = 0;
      for (int p = 0; p < k; ++p)
        if ((c >> p) & 1) o |= 1ull << op.q[k - 1 - p];
      return o;
    };
    if (op.type == OP_X) {
      const uint64_t i1 = base | (1ull << op.q[0]);
      V2<Real> t = sm[base];
      sm[base] = sm[i1];
      sm[i1] = t;
      continue;
    }
    V2<Real> x[32];
    for (uint32_t c = 0; c < dim; ++c) x[c] = sm[base | off(c)];
    for (uint32_t r = 0; r < dim; ++r) {
      V2<Real> acc = mk<Real>(0, 0);
      for (uint32_t c = 0; c < dim; ++c) acc = cadd<Real>(acc, cmul<Real>(ld_coef<Real>(m + r * dim + c), x[c]));
      sm[base | off(r)] = acc;
    }
  }
}

template <typename Real>
__global__ void __launch_bounds__(512) smem_kernel(V2<Real>* __restrict__ amps, uint32_t n, const Op* __restrict__ ops,
                                                   uint32_t op_count, const V2<Real>* __restrict__ coef,
                                                   const PolyTables poly) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V2<Real>* sm = reinterpret_cast<V2<Real>*>(smem_raw);
  const uint64_t len = 1ull << n;
  for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) sm[i] = ld_amp<Real>(amps + i);
  __syncthreads();
  for (uint32_t o = 0; o < op_count; ++o) {
    const Op op = ops[o];
    smem_apply_op<Real>(sm, n, op, coef, poly);
    __syncthreads();
  }
  for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) st_amp<Real>(amps + i, sm[i]);
}

cudaError_t launch_smem_pass(void* amps, int precision, uint32_t n, const Op* ops, uint32_t op_count,
                             const void* coef, PolyTables poly, cudaStream_t s) {
  if (n > 12) return cudaErrorInvalidValue;
  const size_t bytes = (precision == ALEPH_B200_F64 ? 16 : 8) << n;
  if (precision == ALEPH_B200_F64) {
    if (bytes > 48 * 1024)
      cudaFuncSetAttribute(smem_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    smem_kernel<double><<<1, 512, bytes, s>>>((double2*)amps, n, ops, op_count, (const double2*)coef, poly);
  } else {
    if (bytes > 48 * 1024)
      cudaFuncSetAttribute(smem_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    smem_kernel<float><<<1, 512, bytes, s>>>((float2*)amps, n, ops, op_count, (const float2*)coef, poly);
  }
  return cudaGetLastError();
}

// ---- dense k-qubit op on arbitrary qubits (UnitaryKq, k = 3..5) --------------
// One thread per group of 2^K amplitudes (the K target bits varied, the rest
// fixed); consecutive threads take consecutive groups, so every load and store
// is coalesced along the lowest non-target qubits. K is a template parameter:
// the group stays in registers and the 2^K x 2^K product unrolls (the matrix
// is read from shared memory as warp-uniform broadcasts).
template <typename Real, int K>
__global__ void __launch_bounds__(256) kq_kernel(V2<Real>* __restrict__ amps, uint32_t n, const Op* __restrict__ op_p,
                                                 const V2<Real>* __restrict__ coef) {
  constexpr uint32_t DIM = 1u << K;
  __shared__ V2<Real> msm[DIM * DIM];
  __shared__ uint64_t offs[DIM];
  const Op op = *op_p;
  for (uint32_t i = threadIdx.x; i < DIM * DIM; i += blockDim.x) msm[i] = ld_coef<Real>(coef + op.coef + i);
  if (threadIdx.x < DIM) {
    uint64_t o = 0;
#pragma unroll
    for (int p = 0; p < K; ++p)
      if ((threadIdx.x >> p) & 1) o |= 1ull << op.q[K - 1 - p];
    offs[threadIdx.x] = o;
  }
  __syncthreads();
  uint32_t sorted[K];
#pragma unroll
  for (int i = 0; i < K; ++i) sorted[i] = op.q[i];
#pragma unroll
  for (int i = 1; i < K; ++i)
#pragma unroll
    for (int j = i; j > 0; --j)
      if (sorted[j - 1] > sorted[j]) {
        const uint32_t t = sorted[j];
        sorted[j] = sorted[j - 1];
        sorted[j - 1] = t;
      }
  const uint64_t groups = 1ull << (n - K);
  for (uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < groups;
       gi += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = gi;
#pragma unroll
    for (int i = 0; i < K; ++i) base = insert_zero(base, sorted[i]);
    if ((base & op.ctrl) != op.ctrl) continue;
    V2<Real> x[DIM];
#pragma unroll
    for (uint32_t c = 0; c < DIM; ++c) x[c] = ld_amp<Real>(amps + (base | offs[c]));
#pragma unroll
    for (uint32_t r = 0; r < DIM; ++r) {
      V2<Real> acc = mk<Real>(0, 0);
#pragma unroll
      for (uint32_t c = 0; c < DIM; ++c) acc = cadd<Real>(acc, cmul<Real>(msm[r * DIM + c], x[c]));
      st_amp<Real>(amps + (base | offs[r]), acc);
    }
  }
}

template <typename Real>
cudaError_t launch_kq_typed(V2<Real>* amps, uint32_t n, const Op* op_dev, uint32_t k, const V2<Real>* coef,
                            unsigned blocks, cudaStream_t s) {
  switch (k) {
    case 3: kq_kernel<Real, 3><<<blocks, 256, 0, s>>>(amps, n, op_dev, coef); break;
    case 4: kq_kernel<Real, 4><<<blocks, 256, 0, s>>>(amps, n, op_dev, coef); break;
    case 5: kq_kernel<Real, 5><<<blocks, 256, 0, s>>>(amps, n, op_dev, coef); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_kq_pass(void* amps, int precision, uint32_t n, const Op* op_dev, const Op& op_host,
                           const void* coef, cudaStream_t s) {
  if (op_host.nq < 3 || op_host.nq > 5 || n < op_host.nq) return cudaErrorInvalidValue;
  const uint64_t groups = 1ull << (n - op_host.nq);
  const uint64_t blocks64 = (groups + 255) / 256;
  const unsigned blocks = (unsigned)(blocks64 > 148ull * 16 ? 148ull * 16 : blocks64);
  if (precision == ALEPH_B200_F64)
    return launch_kq_typed<double>((double2*)amps, n, op_dev, op_host.nq, (const double2*)coef, blocks, s);
  return launch_kq_typed<float>((float2*)amps, n, op_dev, op_host.nq, (const float2*)coef, blocks, s);
}

// ---- state initialisation / conversion / permutation ------------------------
template <typename Real>
__global__ void init_zero_kernel(V2<Real>* amps, uint64_t len) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x)
    st_amp<Real>(amps + i, mk<Real>(i == 0 ? 1 : 0, 0));
}

cudaError_t launch_init_zero_state(void* amps, uint32_t n, int precision, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  const uint64_t b = (len + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : b);
  if (precision == ALEPH_B200_F64) init_zero_kernel<double><<<blocks, 256, 0, s>>>((double2*)amps, len);
  else init_zero_kernel<float><<<blocks, 256, 0, s>>>((float2*)amps, len);
  return cudaGetLastError();
}

template <typename RS, typename RD>
__global__ void convert_kernel(const V2<RS>* src, V2<RD>* dst, uint64_t count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const V2<RS> a = src[i];
    dst[i] = mk<RD>((RD)a.x, (RD)a.y);
  }
}

cudaError_t launch_convert(const void* src, int sp, void* dst, int dp, uint64_t count, cudaStream_t s) {
  const uint64_t b = (count + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : (b ? b : 1));
  const bool s64 = sp == ALEPH_B200_F64, d64 = dp == ALEPH_B200_F64;
  if (s64 && d64) convert_kernel<double, double><<<blocks, 256, 0, s>>>((const double2*)src, (double2*)dst, count);
  else if (s64) convert_kernel<double, float><<<blocks, 256, 0, s>>>((const double2*)src, (float2*)dst, count);
  else if (d64) convert_kernel<float, double><<<blocks, 256, 0, s>>>((const float2*)src, (double2*)dst, count);
  else convert_kernel<float, float><<<blocks, 256, 0, s>>>((const float2*)src, (float2*)dst, count);
  return cudaGetLastError();
}

// ---- in-place qubit permutation (an involution sigma of the positions) ------
// psi(j) -> psi(sigma(j)). Used for relabelled SWAP networks and for
// unpermute_state (bit_permute_buf, crates/aleph-core/src/perm.rs:25-40, as at
// most two such passes).
//
// Tiles: the tile bits T are the lane qubits 0..4, their images under sigma,
// and further sigma-closed qubits up to 10 bits; the outer bits O are the
// rest, also sigma-closed. Outer value h maps to outer value sigma(h), so a
// CTA takes the pair (h, sigma(h)) at its smaller member, stages both tiles
// in shared memory and writes each into the other with the tile-local
// permutation applied. Global reads and writes run along qubits 0..4
// (32-amplitude runs); shared memory is XOR-swizzled so that reads at the
// permuted local index stay conflict-free.
namespace perm {

// A tile is 2^tile_bits amplitudes: qubits 0..RB-1 (runs of 2^RB contiguous
// amplitudes), their images under sigma, then fixed points and transposed
// pairs up to 2*RB bits. RB = 6 (1 KiB FP64 runs, 4096-amplitude tiles) for
// n >= 12; RB = 5 below. Local index o = column (bits 0..RB-1) | row << RB.
template <int RB>
struct Geometry {
  static constexpr int W = 1 << RB;
  uint32_t tile_bits;                 // |T|
  uint32_t n_outer;                   // |O|
  uint32_t local_identity;            // sigma fixes every tile bit: self-mapped tiles stay put
  uint8_t ob[kMaxQubits];             // outer positions, ascending
  uint8_t osig[kMaxQubits];           // index in ob of sigma(ob[m])
  uint64_t dep_hi[W];                 // global offset of a row's local bits
  // shared-memory slots: a tile amplitude o sits at slot o ^ wr_hi[row(o)]
  // (a per-row XOR of the column), and the amplitude that replaces it comes
  // from slot rd_lo[col(o)] ^ rd_hi[row(o)] (the swizzled slot of sigma(o))
  uint16_t wr_hi[W], rd_lo[W], rd_hi[W];
};

// Work item: an outer value h that owns a pair, or a self-mapped tile that moves.
struct Item {
  uint64_t h, b1, b2;
  bool pair;
};

// This lane's outer bit m = lane (n_outer <= 31): its positions under h, in
// sigma(h) (compact) and in the partner tile's base offset.
struct LaneBit {
  bool act;
  uint32_t m, to_h2, to_b1, to_b2;
};

__device__ __forceinline__ uint64_t or_across_warp(uint64_t x) {
  const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)x);
  const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(x >> 32));
  return (uint64_t)hi << 32 | lo;
}

// Every warp decodes h with one lane per outer bit (no per-thread bit loop).
__device__ __forceinline__ Item next_item(uint32_t local_identity, const LaneBit& lb, uint64_t h, uint64_t nh) {
  for (; h < nh; h += gridDim.x) {
    const uint64_t bit = lb.act ? (h >> lb.m) & 1ull : 0ull;
    const uint64_t h2 = or_across_warp(bit << lb.to_h2);
    if (h2 < h) continue;                   // the pair belongs to its smaller member
    if (h2 == h && local_identity) continue;  // a fixed tile: nothing moves
    return Item{h, or_across_warp(bit << lb.to_b1), or_across_warp(bit << lb.to_b2), h2 != h};
  }
  return Item{nh, 0, 0, false};
}

// Software pipeline: the next item's loads are issued once the current item
// sits in shared memory, and are in flight during its write-back. Each thread
// owns one column (o & (W-1) is fixed, THREADS is a multiple of W), so rows
// are warp-uniform: the row tables are uniform parameter reads.
template <typename Real, int RB, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) permute_kernel(V2<Real>* __restrict__ X, const Geometry<RB> g) {
  constexpr uint32_t W = 1u << RB;
  constexpr int PER_THREAD = (1 << (2 * RB)) / THREADS;
  constexpr uint32_t ROWS_PER_STEP = THREADS / W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V2<Real>* S1 = reinterpret_cast<V2<Real>*>(smem_raw);
  const uint32_t T = 1u << g.tile_bits;
  V2<Real>* S2 = S1 + T;
  const uint64_t nh = 1ull << g.n_outer;
  // lane-indexed parameters are read once (a lane-divergent read of the
  // parameter bank serialises across the warp)
  const uint32_t lane = threadIdx.x & 31u;
  LaneBit lb;
  lb.m = lane;
  lb.act = lane < g.n_outer;
  lb.to_h2 = lb.act ? g.osig[lane] : 0u;
  lb.to_b1 = lb.act ? g.ob[lane] : 0u;
  lb.to_b2 = lb.act ? g.ob[g.osig[lane]] : 0u;
  const uint32_t col = threadIdx.x & (W - 1u);
  const uint32_t row0 = threadIdx.x / W;
  const uint32_t rd_col = g.rd_lo[col];
  V2<Real> r1[PER_THREAD], r2[PER_THREAD];
  auto load = [&](const Item& it) {
#pragma unroll
    for (int k = 0; k < PER_THREAD; ++k) {
      const uint32_t row = row0 + (uint32_t)k * ROWS_PER_STEP;
      if (((row << RB) | col) < T) {
        const uint64_t off = col | g.dep_hi[row];
        r1[k] = X[it.b1 + off];
        if (it.pair) r2[k] = X[it.b2 + off];
      }
    }
  };
  Item cur = next_item(g.local_identity, lb, blockIdx.x, nh);
  if (cur.h >= nh) return;
  load(cur);
  for (;;) {
    __syncthreads();  // the previous write-back is done reading shared memory
#pragma unroll
    for (int k = 0; k < PER_THREAD; ++k) {
      const uint32_t row = row0 + (uint32_t)k * ROWS_PER_STEP;
      if (((row << RB) | col) < T) {
        const uint32_t slot = (row << RB) | (col ^ g.wr_hi[row]);
        S1[slot] = r1[k];
        if (cur.pair) S2[slot] = r2[k];
      }
    }
    __syncthreads();
    const Item nxt = next_item(g.local_identity, lb, cur.h + gridDim.x, nh);
    if (nxt.h < nh) load(nxt);
#pragma unroll
    for (int k = 0; k < PER_THREAD; ++k) {
      const uint32_t row = row0 + (uint32_t)k * ROWS_PER_STEP;
      if (((row << RB) | col) < T) {
        const uint32_t s = rd_col ^ g.rd_hi[row];
        const uint64_t off = col | g.dep_hi[row];
        X[cur.b1 + off] = cur.pair ? S2[s] : S1[s];
        if (cur.pair) X[cur.b2 + off] = S1[s];
      }
    }
    if (nxt.h >= nh) break;
    cur = nxt;
  }
}

// Tile geometry of an involution (host side). `bank_bits`: the column bits
// whose lanes share one shared-memory wavefront (3 for 16-byte amplitudes,
// 4 for 8-byte ones); the row swizzle sends the rows that those lanes read
// after sigma to distinct bank groups.
template <int RB>
static Geometry<RB> geometry(uint32_t n, const uint8_t* sigma, uint32_t bank_bits) {
  constexpr uint32_t W = 1u << RB;
  Geometry<RB> g;
  std::memset(&g, 0, sizeof(g));
  const uint32_t nl = n < (uint32_t)RB ? n : (uint32_t)RB;
  const uint32_t want = n < 2u * RB ? n : 2u * RB;
  uint64_t T = 0;
  for (uint32_t q = 0; q < nl; ++q) T |= (1ull << q) | (1ull << sigma[q]);
  auto count = [&]() { return (uint32_t)__builtin_popcountll(T); };
  for (uint32_t q = 0; q < n && count() < want; ++q)  // fixed points first
    if (!((T >> q) & 1) && sigma[q] == q) T |= 1ull << q;
  for (uint32_t q = 0; q < n && count() + 2 <= want; ++q)  // then transposed pairs
    if (!((T >> q) & 1)) T |= (1ull << q) | (1ull << sigma[q]);
  uint8_t tb[kMaxQubits], local_of[kMaxQubits], outer_of[kMaxQubits];
  uint32_t k = 0, m = 0;
  for (uint32_t q = 0; q < n; ++q) {
    if ((T >> q) & 1) {
      local_of[q] = (uint8_t)k;
      tb[k++] = (uint8_t)q;
    } else {
      outer_of[q] = (uint8_t)m;
      g.ob[m++] = (uint8_t)q;
    }
  }
  g.tile_bits = k;
  g.n_outer = m;
  g.local_identity = 1;
  for (uint32_t j = 0; j < k; ++j) g.local_identity &= sigma[tb[j]] == tb[j] ? 1u : 0u;
  for (uint32_t j = 0; j < m; ++j) g.osig[j] = outer_of[sigma[g.ob[j]]];
  // local sigma as a bit map of the tile index
  uint32_t lsig[2 * RB] = {};
  for (uint32_t j = 0; j < k; ++j) lsig[j] = local_of[sigma[tb[j]]];
  // row swizzle: a linear map M from row bits to column bits. Lane bit b < bank_bits
  // (a column bit) reads local bit lsig[b]; when that is a row bit, M sends it to
  // a bank bit not yet taken, so the 2^bank_bits lanes of a wavefront hit
  // distinct bank groups.
  uint32_t Mrow[RB] = {};
  uint32_t used = 0;
  for (uint32_t b = 0; b < bank_bits && b < k; ++b)
    if (lsig[b] < (uint32_t)RB && lsig[b] < bank_bits) used |= 1u << lsig[b];
  for (uint32_t b = 0; b < bank_bits && b < k; ++b) {
    if (lsig[b] < (uint32_t)RB) continue;
    uint32_t free_bit = 0;
    while (free_bit < bank_bits && ((used >> free_bit) & 1)) ++free_bit;
    if (free_bit == bank_bits) break;
    Mrow[lsig[b] - RB] = 1u << free_bit;
    used |= 1u << free_bit;
  }
  auto M = [&](uint32_t row) {
    uint32_t x = 0;
    for (uint32_t r = 0; r < (uint32_t)RB; ++r)
      if ((row >> r) & 1) x ^= Mrow[r];
    return x;
  };
  auto sig_local = [&](uint32_t o) {
    uint32_t x = 0;
    for (uint32_t j = 0; j < k; ++j)
      if ((o >> j) & 1) x |= 1u << lsig[j];
    return x;
  };
  auto slot = [&](uint32_t o) { return o ^ M(o >> RB); };
  for (uint32_t x = 0; x < W; ++x) {
    uint64_t dep = 0;
    for (uint32_t b = 0; b < (uint32_t)RB; ++b)
      if (((x >> b) & 1) && RB + b < k) dep |= 1ull << tb[RB + b];
    g.dep_hi[x] = dep;
    g.wr_hi[x] = (uint16_t)M(x);
    // slot(sig(o)) is linear in o: split into its column and row parts
    g.rd_lo[x] = (uint16_t)(x < (1u << k) ? slot(sig_local(x)) : 0u);
    g.rd_hi[x] = (uint16_t)((x << RB) < (1u << k) ? slot(sig_local(x << RB)) : 0u);
  }
  return g;
}

template <typename Real, int RB, int THREADS, int MINB>
static cudaError_t launch_rb(void* amps, uint32_t n, const uint8_t* sigma, int sm_count, cudaStream_t s) {
  const uint32_t bank_bits = sizeof(V2<Real>) == 16 ? 3u : 4u;
  const Geometry<RB> g = geometry<RB>(n, sigma, bank_bits);
  if (g.n_outer > 31) return cudaErrorInvalidValue;  // one lane per outer bit
  const uint64_t nh = 1ull << g.n_outer;
  const size_t shm = 2 * ((size_t)1 << g.tile_bits) * sizeof(V2<Real>);
  constexpr size_t kMaxShm = 2 * ((size_t)1 << (2 * RB)) * sizeof(V2<Real>);
  auto kern = permute_kernel<Real, RB, THREADS, MINB>;
  // a persistent grid: exactly the CTAs that are resident at once
  static int resident = 0;
  if (!resident) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxShm);
    if (e != cudaSuccess) return e;
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, THREADS, kMaxShm);
    if (e != cudaSuccess) return e;
    resident = nb > 0 ? nb : 1;
  }
  const uint64_t want = (uint64_t)(sm_count > 0 ? sm_count : 148) * (uint64_t)resident;
  const unsigned blocks = (unsigned)(nh < want ? nh : want);
  kern<<<blocks, THREADS, shm, s>>>((V2<Real>*)amps, g);
  return cudaGetLastError();
}

}  // namespace perm

cudaError_t launch_permute_pass(void* amps, int precision, uint32_t n, const uint8_t* sigma, int sm_count,
                                cudaStream_t s) {
  // 32-amplitude runs and 1024-amplitude tiles: a tile pair is 32 KiB of
  // shared memory in FP64, so several CTAs share an SM and cover each other's
  // barrier bubbles. (64-amplitude runs need a 128 KiB pair, one CTA per SM:
  // slower on B200 for every permutation measured, 2.4-3.1 against
  // 3.7-5.5 TB/s in FP64.)
  if (precision == ALEPH_B200_F64) return perm::launch_rb<double, 5, 256, 1>(amps, n, sigma, sm_count, s);
  return perm::launch_rb<float, 5, 256, 1>(amps, n, sigma, sm_count, s);
}

// ---- renormalisation (end of a tensor-core gate stream) ----------------------
// Tensor-core FP32 accumulation drifts the state norm systematically (by
// ~1e-6 per block pass); one FP64 norm reduction and one rescale pass restore
// |psi| = 1 without a host round trip.
template <typename Real>
__global__ void rescale_kernel(V2<Real>* __restrict__ amps, uint64_t len, const double* __restrict__ norm2) {
  const double s = norm2[0] > 0.0 ? rsqrt(norm2[0]) : 1.0;
  // four independent loads per step (bytes in flight, as in norm_kernel)
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < len; i += 4 * stride) {
    V2<Real> a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = ld_amp<Real>(amps + i + k * stride);
#pragma unroll
    for (int k = 0; k < 4; ++k) st_amp<Real>(amps + i + k * stride, mk<Real>((Real)(a[k].x * s), (Real)(a[k].y * s)));
  }
  for (; i < len; i += stride) {
    const V2<Real> a = ld_amp<Real>(amps + i);
    st_amp<Real>(amps + i, mk<Real>((Real)(a.x * s), (Real)(a.y * s)));
  }
}

cudaError_t launch_rescale(void* amps, int precision, uint32_t n, const double* norm2, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  const uint64_t b = (len + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : b);
  if (precision == ALEPH_B200_F64) rescale_kernel<double><<<blocks, 256, 0, s>>>((double2*)amps, len, norm2);
  else rescale_kernel<float><<<blocks, 256, 0, s>>>((float2*)amps, len, norm2);
  return cudaGetLastError();
}

cudaError_t launch_renormalize(void* amps, int precision, uint32_t n, double* partials, uint32_t nblocks, double* out2,
                               cudaStream_t s) {
  cudaError_t e = launch_norm(amps, precision, n, partials, nblocks, out2, s);
  if (e != cudaSuccess) return e;
  const uint64_t len = 1ull << n;
  const uint64_t b = (len + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : b);
  if (precision == ALEPH_B200_F64) rescale_kernel<double><<<blocks, 256, 0, s>>>((double2*)amps, len, out2);
  else rescale_kernel<float><<<blocks, 256, 0, s>>>((float2*)amps, len, out2);
  return cudaGetLastError();
}

}  // namespace ab
