// kernels_gates.cu — CUDA-core gate passes of the B200 state-vector engine.
//
// * tile_kernel: the warp-tile pass. One warp owns a tile of 2^(5+R)
//   amplitudes: lane bits = qubits 0..4 (so every load/store instruction of a
//   warp moves 32 consecutive amplitudes — 512 B in FP64, 256 B in FP32) and
//   each thread keeps 2^R amplitudes in registers, spanning the R "register"
//   qubits of the pass. An ordered list of ops is applied in registers: gates
//   on register qubits are pure register arithmetic, gates on qubits 0..4 use
//   warp shuffles, diagonal ops (CZ, phases, DiagonalPhase) act on any qubit
//   from the amplitude's global index, and controls may sit on any qubit. One
//   HBM read + one write per pass, however many gates it applies.
// * smem_kernel: states with n <= 12 run the whole op list in one CTA with
//   the state resident in shared memory.
// * kq_kernel: dense k-qubit (k = 3..5) UnitaryKq on arbitrary qubits.
//
// Semantics follow the reference kernels: pair/quartet butterflies
// (crates/aleph-sv/src/kernels/aos.rs:192-223, :1335-1394), MSB-first operand
// order (crates/aleph-sv/src/kernels/unitary_kq.rs:66-96), controls as an AND
// mask over the basis index (aos.rs:198-205).

#include <cstdio>

#include "common.cuh"

namespace ab {

constexpr unsigned FULL = 0xffffffffu;

template <int R>
__device__ __forceinline__ uint64_t roff(int r, const uint64_t (&hb)[5]) {
  uint64_t o = 0;
#pragma unroll
  for (int j = 0; j < R; ++j)
    if ((r >> j) & 1) o |= hb[j];
  return o;
}

// ---- register-qubit ops -----------------------------------------------------
template <typename Real, int R, int J>
__device__ __forceinline__ void reg_1q(V2<Real> (&v)[1 << R], const V2<Real>* m, uint64_t ctrl, uint64_t gl,
                                       const uint64_t (&hb)[5]) {
  const V2<Real> m0 = ld_coef<Real>(m), m1 = ld_coef<Real>(m + 1), m2 = ld_coef<Real>(m + 2),
                 m3 = ld_coef<Real>(m + 3);
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (1 << J)) continue;
    const int r1 = r | (1 << J);
    if (ctrl && (((gl | roff<R>(r, hb)) & ctrl) != ctrl)) continue;
    const V2<Real> a = v[r], b = v[r1];
    v[r] = cmul2<Real>(m0, a, m1, b);
    v[r1] = cmul2<Real>(m2, a, m3, b);
  }
}

template <typename Real, int R, int J>
__device__ __forceinline__ void reg_x(V2<Real> (&v)[1 << R], uint64_t ctrl, uint64_t gl, const uint64_t (&hb)[5]) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (1 << J)) continue;
    const int r1 = r | (1 << J);
    if (ctrl && (((gl | roff<R>(r, hb)) & ctrl) != ctrl)) continue;
    const V2<Real> t = v[r];
    v[r] = v[r1];
    v[r1] = t;
  }
}

// 4x4 on register bits JA (matrix MSB) and JB (matrix LSB), JA != JB.
template <typename Real, int R, int JA, int JB>
__device__ __forceinline__ void reg_2q(V2<Real> (&v)[1 << R], const V2<Real>* m, uint64_t ctrl, uint64_t gl,
                                       const uint64_t (&hb)[5]) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & ((1 << JA) | (1 << JB))) continue;
    if (ctrl && (((gl | roff<R>(r, hb)) & ctrl) != ctrl)) continue;
    const int idx[4] = {r, r | (1 << JB), r | (1 << JA), r | (1 << JA) | (1 << JB)};
    V2<Real> x[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = v[idx[c]];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      V2<Real> acc = cmul2<Real>(ld_coef<Real>(m + 4 * k), x[0], ld_coef<Real>(m + 4 * k + 1), x[1]);
      acc = cadd<Real>(acc, cmul2<Real>(ld_coef<Real>(m + 4 * k + 2), x[2], ld_coef<Real>(m + 4 * k + 3), x[3]));
      v[idx[k]] = acc;
    }
  }
}

// ---- lane-qubit ops (qubits 0..4, warp shuffles) ----------------------------
template <typename Real, int R>
__device__ __forceinline__ void lane_1q(V2<Real> (&v)[1 << R], int s, const V2<Real>* m, uint64_t ctrl, uint64_t gl,
                                        const uint64_t (&hb)[5]) {
  const int lane = threadIdx.x & 31;
  const bool hi = (lane >> s) & 1;
  const V2<Real> cs = ld_coef<Real>(m + (hi ? 3 : 0));  // coefficient on own amplitude
  const V2<Real> co = ld_coef<Real>(m + (hi ? 2 : 1));  // coefficient on partner amplitude
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    const V2<Real> o = shfl_xor<Real>(v[r], 1 << s);
    const V2<Real> nv = cmul2<Real>(cs, v[r], co, o);
    if (!ctrl || (((gl | roff<R>(r, hb)) & ctrl) == ctrl)) v[r] = nv;
  }
}

template <typename Real, int R>
__device__ __forceinline__ void lane_x(V2<Real> (&v)[1 << R], int s, uint64_t ctrl, uint64_t gl,
                                       const uint64_t (&hb)[5]) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    const V2<Real> o = shfl_xor<Real>(v[r], 1 << s);
    if (!ctrl || (((gl | roff<R>(r, hb)) & ctrl) == ctrl)) v[r] = o;
  }
}

// 4x4 with matrix MSB on register bit JA and LSB on lane bit s.
template <typename Real, int R, int JA>
__device__ __forceinline__ void regl_2q(V2<Real> (&v)[1 << R], int s, const V2<Real>* m, uint64_t ctrl, uint64_t gl,
                                        const uint64_t (&hb)[5]) {
  const int lane = threadIdx.x & 31;
  const int l = (lane >> s) & 1;
  V2<Real> r0[4], r1[4];  // own rows: k = l and k = 2 + l
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    r0[c] = ld_coef<Real>(m + 4 * l + c);
    r1[c] = ld_coef<Real>(m + 4 * (2 + l) + c);
  }
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (1 << JA)) continue;
    const int ra = r | (1 << JA);
    const V2<Real> A0 = v[r], A1 = v[ra];
    const V2<Real> P0 = shfl_xor<Real>(A0, 1 << s), P1 = shfl_xor<Real>(A1, 1 << s);
    if (ctrl && (((gl | roff<R>(r, hb)) & ctrl) != ctrl)) continue;
    const V2<Real> x0 = l ? P0 : A0, x1 = l ? A0 : P0, x2 = l ? P1 : A1, x3 = l ? A1 : P1;
    v[r] = cadd<Real>(cmul2<Real>(r0[0], x0, r0[1], x1), cmul2<Real>(r0[2], x2, r0[3], x3));
    v[ra] = cadd<Real>(cmul2<Real>(r1[0], x0, r1[1], x1), cmul2<Real>(r1[2], x2, r1[3], x3));
  }
}

// 4x4 with matrix MSB on lane bit sa and LSB on lane bit sb.
template <typename Real, int R>
__device__ __forceinline__ void lane_2q(V2<Real> (&v)[1 << R], int sa, int sb, const V2<Real>* m, uint64_t ctrl,
                                        uint64_t gl, const uint64_t (&hb)[5]) {
  const int lane = threadIdx.x & 31;
  const int k0 = (((lane >> sa) & 1) << 1) | ((lane >> sb) & 1);
  const V2<Real> c0 = ld_coef<Real>(m + 4 * k0 + k0), c1 = ld_coef<Real>(m + 4 * k0 + (k0 ^ 1)),
                 c2 = ld_coef<Real>(m + 4 * k0 + (k0 ^ 2)), c3 = ld_coef<Real>(m + 4 * k0 + (k0 ^ 3));
  const int mb = 1 << sb, ma = 1 << sa;
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    const V2<Real> own = v[r];
    const V2<Real> p1 = shfl_xor<Real>(own, mb), p2 = shfl_xor<Real>(own, ma), p3 = shfl_xor<Real>(own, ma | mb);
    const V2<Real> nv = cadd<Real>(cmul2<Real>(c0, own, c1, p1), cmul2<Real>(c2, p2, c3, p3));
    if (!ctrl || (((gl | roff<R>(r, hb)) & ctrl) == ctrl)) v[r] = nv;
  }
}

template <typename Real, int R>
__device__ __forceinline__ void dispatch_reg_1q(int J, V2<Real> (&v)[1 << R], const V2<Real>* m, uint64_t ctrl,
                                                uint64_t gl, const uint64_t (&hb)[5]) {
  switch (J) {
    case 0: if constexpr (R > 0) reg_1q<Real, R, 0>(v, m, ctrl, gl, hb); break;
    case 1: if constexpr (R > 1) reg_1q<Real, R, 1>(v, m, ctrl, gl, hb); break;
    case 2: if constexpr (R > 2) reg_1q<Real, R, 2>(v, m, ctrl, gl, hb); break;
    case 3: if constexpr (R > 3) reg_1q<Real, R, 3>(v, m, ctrl, gl, hb); break;
    case 4: if constexpr (R > 4) reg_1q<Real, R, 4>(v, m, ctrl, gl, hb); break;
  }
}
template <typename Real, int R>
__device__ __forceinline__ void dispatch_reg_x(int J, V2<Real> (&v)[1 << R], uint64_t ctrl, uint64_t gl,
                                               const uint64_t (&hb)[5]) {
  switch (J) {
    case 0: if constexpr (R > 0) reg_x<Real, R, 0>(v, ctrl, gl, hb); break;
    case 1: if constexpr (R > 1) reg_x<Real, R, 1>(v, ctrl, gl, hb); break;
    case 2: if constexpr (R > 2) reg_x<Real, R, 2>(v, ctrl, gl, hb); break;
    case 3: if constexpr (R > 3) reg_x<Real, R, 3>(v, ctrl, gl, hb); break;
    case 4: if constexpr (R > 4) reg_x<Real, R, 4>(v, ctrl, gl, hb); break;
  }
}
template <typename Real, int R>
__device__ __forceinline__ void dispatch_regl_2q(int JA, int s, V2<Real> (&v)[1 << R], const V2<Real>* m,
                                                 uint64_t ctrl, uint64_t gl, const uint64_t (&hb)[5]) {
  switch (JA) {
    case 0: if constexpr (R > 0) regl_2q<Real, R, 0>(v, s, m, ctrl, gl, hb); break;
    case 1: if constexpr (R > 1) regl_2q<Real, R, 1>(v, s, m, ctrl, gl, hb); break;
    case 2: if constexpr (R > 2) regl_2q<Real, R, 2>(v, s, m, ctrl, gl, hb); break;
    case 3: if constexpr (R > 3) regl_2q<Real, R, 3>(v, s, m, ctrl, gl, hb); break;
    case 4: if constexpr (R > 4) regl_2q<Real, R, 4>(v, s, m, ctrl, gl, hb); break;
  }
}
template <typename Real, int R>
__device__ __forceinline__ void dispatch_reg_2q(int JA, int JB, V2<Real> (&v)[1 << R], const V2<Real>* m,
                                                uint64_t ctrl, uint64_t gl, const uint64_t (&hb)[5]) {
#define AB_RR(a, b)                                          \
  case (a)*8 + (b):                                          \
    if constexpr (R > (a) && R > (b) && (a) != (b))          \
      reg_2q<Real, R, (a), (b)>(v, m, ctrl, gl, hb);         \
    break;
  switch (JA * 8 + JB) {
    AB_RR(0, 1) AB_RR(0, 2) AB_RR(0, 3) AB_RR(0, 4)
    AB_RR(1, 0) AB_RR(1, 2) AB_RR(1, 3) AB_RR(1, 4)
    AB_RR(2, 0) AB_RR(2, 1) AB_RR(2, 3) AB_RR(2, 4)
    AB_RR(3, 0) AB_RR(3, 1) AB_RR(3, 2) AB_RR(3, 4)
    AB_RR(4, 0) AB_RR(4, 1) AB_RR(4, 2) AB_RR(4, 3)
  }
#undef AB_RR
}

// ---- the warp-tile pass -----------------------------------------------------
template <typename Real, int R>
__global__ void __launch_bounds__(128) tile_kernel(V2<Real>* __restrict__ amps, const TilePass p,
                                                   const Op* __restrict__ ops, const V2<Real>* __restrict__ coef,
                                                   const PolyTables poly) {
  constexpr int NR = 1 << R;
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (warp >= (1ull << (p.n - 5 - R))) return;

  uint64_t hb[5] = {0, 0, 0, 0, 0};
  uint64_t tilemask = 0x1Full;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    hb[j] = 1ull << p.hq[j];
    tilemask |= hb[j];
  }
  // Deposit the warp index into the non-tile qubits (ascending).
  uint64_t base = 0, w = warp;
  for (uint32_t pos = 5; w != 0 && pos < p.n; ++pos) {
    if ((tilemask >> pos) & 1) continue;
    base |= (w & 1ull) << pos;
    w >>= 1;
  }
  const uint64_t gl = base | (uint64_t)lane;

  V2<Real> v[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = ld_amp<Real>(amps + (gl | roff<R>(r, hb)));

  for (uint32_t i = 0; i < p.op_count; ++i) {
    const Op op = ops[p.op_begin + i];
    const V2<Real>* m = coef + op.coef;
    switch (op.type) {
      case OP_1Q:
        if (op.a < 5) lane_1q<Real, R>(v, op.a, m, op.ctrl, gl, hb);
        else dispatch_reg_1q<Real, R>(op.a - 5, v, m, op.ctrl, gl, hb);
        break;
      case OP_X:
        if (op.a < 5) lane_x<Real, R>(v, op.a, op.ctrl, gl, hb);
        else dispatch_reg_x<Real, R>(op.a - 5, v, op.ctrl, gl, hb);
        break;
      case OP_2Q:
        // Planner canonicalises slot a > slot b.
        if (op.b >= 5) dispatch_reg_2q<Real, R>(op.a - 5, op.b - 5, v, m, op.ctrl, gl, hb);
        else if (op.a >= 5) dispatch_regl_2q<Real, R>(op.a - 5, op.b, v, m, op.ctrl, gl, hb);
        else lane_2q<Real, R>(v, op.a, op.b, m, op.ctrl, gl, hb);
        break;
      default:  // diagonal ops on any qubit
#pragma unroll
        for (int r = 0; r < NR; ++r) v[r] = apply_diag_op<Real>(op, v[r], gl | roff<R>(r, hb), coef, poly);
        break;
    }
  }

#pragma unroll
  for (int r = 0; r < NR; ++r) st_amp<Real>(amps + (gl | roff<R>(r, hb)), v[r]);
}

template <typename Real, int R>
static cudaError_t launch_tile_t(void* amps, const TilePass& p, const Op* ops, const void* coef, PolyTables poly,
                                 cudaStream_t s) {
  const uint64_t warps = 1ull << (p.n - 5 - R);
  const uint32_t wpb = 4;
  const uint64_t blocks = (warps + wpb - 1) / wpb;
  tile_kernel<Real, R><<<(unsigned)blocks, 32 * wpb, 0, s>>>((V2<Real>*)amps, p, ops, (const V2<Real>*)coef, poly);
  return cudaGetLastError();
}

cudaError_t launch_tile_pass(void* amps, int precision, const TilePass& p, const Op* ops, const void* coef,
                             PolyTables poly, cudaStream_t s) {
  if (p.R < 1 || p.R > 5 || p.n < 5 + p.R) return cudaErrorInvalidValue;
  const bool f64 = precision == ALEPH_B200_F64;
  switch (p.R) {
    case 1: return f64 ? launch_tile_t<double, 1>(amps, p, ops, coef, poly, s) : launch_tile_t<float, 1>(amps, p, ops, coef, poly, s);
    case 2: return f64 ? launch_tile_t<double, 2>(amps, p, ops, coef, poly, s) : launch_tile_t<float, 2>(amps, p, ops, coef, poly, s);
    case 3: return f64 ? launch_tile_t<double, 3>(amps, p, ops, coef, poly, s) : launch_tile_t<float, 3>(amps, p, ops, coef, poly, s);
    case 4: return f64 ? launch_tile_t<double, 4>(amps, p, ops, coef, poly, s) : launch_tile_t<float, 4>(amps, p, ops, coef, poly, s);
    default: return f64 ? launch_tile_t<double, 5>(amps, p, ops, coef, poly, s) : launch_tile_t<float, 5>(amps, p, ops, coef, poly, s);
  }
}

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
template <typename Real>
__global__ void __launch_bounds__(256) kq_kernel(V2<Real>* __restrict__ amps, uint32_t n, const Op* __restrict__ op_p,
                                                 const V2<Real>* __restrict__ coef) {
  __shared__ V2<Real> msm[32 * 32];
  __shared__ uint64_t offs[32];
  const Op op = *op_p;
  const int k = op.nq;
  const uint32_t dim = 1u << k;
  for (uint32_t i = threadIdx.x; i < dim * dim; i += blockDim.x) msm[i] = ld_coef<Real>(coef + op.coef + i);
  if (threadIdx.x < dim) {
    uint64_t o = 0;
    for (int p = 0; p < k; ++p)
      if ((threadIdx.x >> p) & 1) o |= 1ull << op.q[k - 1 - p];
    offs[threadIdx.x] = o;
  }
  __syncthreads();
  uint32_t sorted[6];
  for (int i = 0; i < k; ++i) sorted[i] = op.q[i];
  for (int i = 1; i < k; ++i)
    for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; --j) {
      uint32_t t = sorted[j];
      sorted[j] = sorted[j - 1];
      sorted[j - 1] = t;
    }
  const uint64_t groups = 1ull << (n - k);
  for (uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < groups;
       gi += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = gi;
    for (int i = 0; i < k; ++i) base = insert_zero(base, sorted[i]);
    if ((base & op.ctrl) != op.ctrl) continue;
    V2<Real> x[32];
    for (uint32_t c = 0; c < dim; ++c) x[c] = ld_amp<Real>(amps + (base | offs[c]));
    for (uint32_t r = 0; r < dim; ++r) {
      V2<Real> acc = mk<Real>(0, 0);
      for (uint32_t c = 0; c < dim; ++c) acc = cadd<Real>(acc, cmul<Real>(msm[r * dim + c], x[c]));
      st_amp<Real>(amps + (base | offs[r]), acc);
    }
  }
}

cudaError_t launch_kq_pass(void* amps, int precision, uint32_t n, const Op* op_dev, const Op& op_host,
                           const void* coef, cudaStream_t s) {
  const uint64_t groups = 1ull << (n - op_host.nq);
  const uint64_t blocks64 = (groups + 255) / 256;
  const unsigned blocks = (unsigned)(blocks64 > 148ull * 16 ? 148ull * 16 : blocks64);
  if (precision == ALEPH_B200_F64)
    kq_kernel<double><<<blocks, 256, 0, s>>>((double2*)amps, n, op_dev, (const double2*)coef);
  else
    kq_kernel<float><<<blocks, 256, 0, s>>>((float2*)amps, n, op_dev, (const float2*)coef);
  return cudaGetLastError();
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

// bit_permute_buf (crates/aleph-core/src/perm.rs:25-40): out[i] = in[j],
// j = sum over logical bits lq of i of (1 << perm[lq]).
template <typename Real>
__global__ void unpermute_kernel(const V2<Real>* __restrict__ src, V2<Real>* __restrict__ dst, uint32_t n,
                                 const uint32_t* __restrict__ perm) {
  const uint64_t len = 1ull << n;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = 0;
    for (uint32_t lq = 0; lq < n; ++lq)
      if ((i >> lq) & 1) j |= 1ull << __ldg(&perm[lq]);
    dst[i] = ld_amp<Real>(src + j);
  }
}

cudaError_t launch_unpermute(const void* src, void* dst, int precision, uint32_t n, const uint32_t* perm_dev,
                             cudaStream_t s) {
  const uint64_t len = 1ull << n;
  const uint64_t b = (len + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : b);
  if (precision == ALEPH_B200_F64)
    unpermute_kernel<double><<<blocks, 256, 0, s>>>((const double2*)src, (double2*)dst, n, perm_dev);
  else
    unpermute_kernel<float><<<blocks, 256, 0, s>>>((const float2*)src, (float2*)dst, n, perm_dev);
  return cudaGetLastError();
}

}  // namespace ab
