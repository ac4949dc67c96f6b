// kernels_tile.cu — the warp-tile gate pass of the B200 state-vector engine.
//
// One warp owns a tile of 2^(5+R) amplitudes: the lane index supplies qubits
// 0..4, so every load/store instruction of a warp moves 32 consecutive
// amplitudes (512 B in FP64, 256 B in FP32, fully coalesced 16-/8-byte
// accesses), and each thread keeps 2^R amplitudes in registers spanning the R
// "register" qubits hq[0..R) of the pass. An ordered op list is applied in
// registers: gates on register qubits are register arithmetic, gates on
// qubits 0..4 use warp shuffles, diagonal ops (CZ, phases, DiagonalPhase) act
// on any qubit, and controls may sit on any qubit. One HBM read and one write
// per pass, however many gates it applies.
//
// Per-element predicates (controls, CZ masks, diagonal table indices) are
// split by the planner into a thread-constant part (bits of the lane and of
// the tile base) and a register part (an R-bit mask tested against the
// compile-time register index), so the inner loops do 32-bit tests only.
//
// Semantics follow the reference kernels: pair/quartet butterflies
// (crates/aleph-sv/src/kernels/aos.rs:192-223, :1335-1394), MSB-first operand
// order (crates/aleph-sv/src/kernels/unitary_kq.rs:66-96), controls as an AND
// mask over the basis index (aos.rs:198-205).

#include "common.cuh"

namespace ab {

template <int R>
__device__ __forceinline__ uint64_t roff(int r, const uint64_t (&hb)[5]) {
  uint64_t o = 0;
#pragma unroll
  for (int j = 0; j < R; ++j)
    if ((r >> j) & 1) o |= hb[j];
  return o;
}

#define AB_ON(r) (thr && (((r) & creg) == creg))

// ---- register-qubit ops -----------------------------------------------------
template <typename Real, int R, int J>
__device__ __forceinline__ void reg_1q(V2<Real> (&v)[1 << R], const V2<Real>* m, bool thr, uint32_t creg) {
  const V2<Real> m0 = ld_coef<Real>(m), m1 = ld_coef<Real>(m + 1), m2 = ld_coef<Real>(m + 2),
                 m3 = ld_coef<Real>(m + 3);
  if (thr && creg == 0) {  // no register-part controls: every pair, no per-pair predicate
#pragma unroll
    for (int r = 0; r < (1 << R); ++r) {
      if (r & (1 << J)) continue;
      const int r1 = r | (1 << J);
      const V2<Real> a = v[r], b = v[r1];
      v[r] = cmul2<Real>(m0, a, m1, b);
      v[r1] = cmul2<Real>(m2, a, m3, b);
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (1 << J)) continue;
    const int r1 = r | (1 << J);
    if (!AB_ON(r)) continue;
    const V2<Real> a = v[r], b = v[r1];
    v[r] = cmul2<Real>(m0, a, m1, b);
    v[r1] = cmul2<Real>(m2, a, m3, b);
  }
}

// Two one-qubit gates in a row, U1 on register bit J1 then U2 on register bit
// J2 != J1, neither controlled: one sweep over quartets. U1 writes four
// temporaries and U2 writes straight back into the loop-carried registers,
// so no amplitude moves between the two gates (a lone gate must park three
// of every four results while its inputs are still live).
template <typename Real, int R, int J1, int J2>
__device__ __forceinline__ void reg_1q_pair(V2<Real> (&v)[1 << R], const V2<Real>* m, const V2<Real>* u) {
  const V2<Real> m0 = ld_coef<Real>(m), m1 = ld_coef<Real>(m + 1), m2 = ld_coef<Real>(m + 2),
                 m3 = ld_coef<Real>(m + 3);
  const V2<Real> u0 = ld_coef<Real>(u), u1 = ld_coef<Real>(u + 1), u2 = ld_coef<Real>(u + 2),
                 u3 = ld_coef<Real>(u + 3);
  constexpr int B1 = 1 << J1, B2 = 1 << J2;
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (B1 | B2)) continue;
    const V2<Real> x00 = v[r], x01 = v[r | B1], x10 = v[r | B2], x11 = v[r | B1 | B2];
    const V2<Real> t00 = cmul2<Real>(m0, x00, m1, x01), t01 = cmul2<Real>(m2, x00, m3, x01);
    const V2<Real> t10 = cmul2<Real>(m0, x10, m1, x11), t11 = cmul2<Real>(m2, x10, m3, x11);
    v[r] = cmul2<Real>(u0, t00, u1, t10);
    v[r | B2] = cmul2<Real>(u2, t00, u3, t10);
    v[r | B1] = cmul2<Real>(u0, t01, u1, t11);
    v[r | B1 | B2] = cmul2<Real>(u2, t01, u3, t11);
  }
}

// Sign flip of the registers r with (r & K) == K: a CZ-like op whose
// register part K is known at compile time runs without per-amplitude tests.
template <typename Real, int R, uint32_t K>
__device__ __forceinline__ void reg_neg(V2<Real> (&v)[1 << R]) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r)
    if (((uint32_t)r & K) == K) v[r] = cneg<Real>(v[r]);
}

template <typename Real, int R>
__device__ __forceinline__ void dispatch_neg(V2<Real> (&v)[1 << R], uint32_t creg) {
#define AB_NEG(k) \
  case k:         \
    if constexpr ((k) < (1u << R)) reg_neg<Real, R, k>(v); \
    break;
  switch (creg) {
    AB_NEG(0) AB_NEG(1) AB_NEG(2) AB_NEG(3) AB_NEG(4) AB_NEG(5) AB_NEG(6) AB_NEG(7)
    AB_NEG(8) AB_NEG(9) AB_NEG(10) AB_NEG(11) AB_NEG(12) AB_NEG(13) AB_NEG(14) AB_NEG(15)
    AB_NEG(16) AB_NEG(17) AB_NEG(18) AB_NEG(19) AB_NEG(20) AB_NEG(21) AB_NEG(22) AB_NEG(23)
    AB_NEG(24) AB_NEG(25) AB_NEG(26) AB_NEG(27) AB_NEG(28) AB_NEG(29) AB_NEG(30) AB_NEG(31)
  }
#undef AB_NEG
}

template <typename Real, int R, int J>
__device__ __forceinline__ void reg_x(V2<Real> (&v)[1 << R], bool thr, uint32_t creg) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & (1 << J)) continue;
    const int r1 = r | (1 << J);
    if (!AB_ON(r)) continue;
    const V2<Real> t = v[r];
    v[r] = v[r1];
    v[r1] = t;
  }
}

// 4x4 on register bits JA (matrix MSB) > JB (matrix LSB).
template <typename Real, int R, int JA, int JB>
__device__ __forceinline__ void reg_2q(V2<Real> (&v)[1 << R], const V2<Real>* m, bool thr, uint32_t creg) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    if (r & ((1 << JA) | (1 << JB))) continue;
    if (!AB_ON(r)) continue;
    const int i0 = r, i1 = r | (1 << JB), i2 = r | (1 << JA), i3 = r | (1 << JA) | (1 << JB);
    const V2<Real> x0 = v[i0], x1 = v[i1], x2 = v[i2], x3 = v[i3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const V2<Real> acc = cadd<Real>(cmul2<Real>(ld_coef<Real>(m + 4 * k), x0, ld_coef<Real>(m + 4 * k + 1), x1),
                                      cmul2<Real>(ld_coef<Real>(m + 4 * k + 2), x2, ld_coef<Real>(m + 4 * k + 3), x3));
      const int dst = k == 0 ? i0 : k == 1 ? i1 : k == 2 ? i2 : i3;
      v[dst] = acc;
    }
  }
}

// The q-th register index with bits JA and JB clear (q's bits deposited in order).
template <int R, int JA, int JB>
__device__ constexpr int quartet_base(int q) {
  int r = 0, bit = 0;
  for (int j = 0; j < R; ++j) {
    if (j == JA || j == JB) continue;
    if ((q >> bit) & 1) r |= 1 << j;
    ++bit;
  }
  return r;
}

// One row of a 4x4: c0 x0 + c1 x1 + c2 x2 + c3 x3 as one multiply-add chain
// per component (1 multiply + 7 fused multiply-adds).
template <typename Real>
__device__ __forceinline__ V2<Real> mac4(V2<Real> c0, V2<Real> x0, V2<Real> c1, V2<Real> x1, V2<Real> c2, V2<Real> x2,
                                         V2<Real> c3, V2<Real> x3) {
  Real re = c0.x * x0.x, im = c0.x * x0.y;
  re = fma(-c0.y, x0.y, re);
  im = fma(c0.y, x0.x, im);
  re = fma(c1.x, x1.x, re);
  im = fma(c1.x, x1.y, im);
  re = fma(-c1.y, x1.y, re);
  im = fma(c1.y, x1.x, im);
  re = fma(c2.x, x2.x, re);
  im = fma(c2.x, x2.y, im);
  re = fma(-c2.y, x2.y, re);
  im = fma(c2.y, x2.x, im);
  re = fma(c3.x, x3.x, re);
  im = fma(c3.x, x3.y, im);
  re = fma(-c3.y, x3.y, re);
  im = fma(c3.y, x3.x, im);
  return mk<Real>(re, im);
}

// Uncontrolled 4x4 on register bits JA (matrix MSB) > JB, QB quartets at a
// time: each row of coefficients is loaded once per QB quartets and the
// block's outputs wait in registers until its inputs are spent. The
// coefficients are uniform across the warp, and with the tile in registers
// they cannot all stay live; loaded per quartet, they were most of the pass's
// L1 traffic.
template <typename Real, int R, int JA, int JB, int QB>
__device__ __forceinline__ void reg_2q_blocked(V2<Real> (&v)[1 << R], const V2<Real>* m) {
  constexpr int NQ = 1 << (R - 2);
  constexpr int A = 1 << JA, B = 1 << JB;
#pragma unroll
  for (int q0 = 0; q0 < NQ; q0 += QB) {
    V2<Real> o[QB][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const V2<Real> c0 = ld_coef<Real>(m + 4 * k), c1 = ld_coef<Real>(m + 4 * k + 1),
                     c2 = ld_coef<Real>(m + 4 * k + 2), c3 = ld_coef<Real>(m + 4 * k + 3);
#pragma unroll
      for (int j = 0; j < QB; ++j) {
        const int r = quartet_base<R, JA, JB>(q0 + j);
        o[j][k] = mac4<Real>(c0, v[r], c1, v[r | B], c2, v[r | A], c3, v[r | A | B]);
      }
    }
#pragma unroll
    for (int j = 0; j < QB; ++j) {
      const int r = quartet_base<R, JA, JB>(q0 + j);
      v[r] = o[j][0];
      v[r | B] = o[j][1];
      v[r | A] = o[j][2];
      v[r | A | B] = o[j][3];
    }
  }
}

// ---- lane-qubit ops (qubits 0..4, warp shuffles) ----------------------------
template <typename Real, int R>
__device__ __forceinline__ void lane_1q(V2<Real> (&v)[1 << R], int s, const V2<Real>* m, bool thr, uint32_t creg) {
  const int lane = threadIdx.x & 31;
  const bool hi = (lane >> s) & 1;
  const V2<Real> cs = ld_coef<Real>(m + (hi ? 3 : 0));  // coefficient on own amplitude
  const V2<Real> co = ld_coef<Real>(m + (hi ? 2 : 1));  // coefficient on partner amplitude
  if (thr && creg == 0) {  // no register-part controls
#pragma unroll
    for (int r = 0; r < (1 << R); ++r) {
      const V2<Real> o = shfl_xor<Real>(v[r], 1 << s);
      v[r] = cmul2<Real>(cs, v[r], co, o);
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    const V2<Real> o = shfl_xor<Real>(v[r], 1 << s);
    const V2<Real> nv = cmul2<Real>(cs, v[r], co, o);
    if (AB_ON(r)) v[r] = nv;
  }
}

template <typename Real, int R>
__device__ __forceinline__ void lane_x(V2<Real> (&v)[1 << R], int s, bool thr, uint32_t creg) {
#pragma unroll
  for (int r = 0; r < (1 << R); ++r) {
    const V2<Real> o = shfl_xor<Real>(v[r], 1 << s);
    if (AB_ON(r)) v[r] = o;
  }
}

// 4x4 with matrix MSB on register bit JA and LSB on lane bit s.
template <typename Real, int R, int JA>
__device__ __forceinline__ void regl_2q(V2<Real> (&v)[1 << R], int s, const V2<Real>* m, bool thr, uint32_t creg) {
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
    if (!AB_ON(r)) continue;
    const V2<Real> x0 = l ? P0 : A0, x1 = l ? A0 : P0, x2 = l ? P1 : A1, x3 = l ? A1 : P1;
    v[r] = cadd<Real>(cmul2<Real>(r0[0], x0, r0[1], x1), cmul2<Real>(r0[2], x2, r0[3], x3));
    v[ra] = cadd<Real>(cmul2<Real>(r1[0], x0, r1[1], x1), cmul2<Real>(r1[2], x2, r1[3], x3));
  }
}

// 4x4 with matrix MSB on lane bit sa and LSB on lane bit sb.
template <typename Real, int R>
__device__ __forceinline__ void lane_2q(V2<Real> (&v)[1 << R], int sa, int sb, const V2<Real>* m, bool thr,
                                        uint32_t creg) {
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
    if (AB_ON(r)) v[r] = nv;
  }
}

// ---- diagonal ops -------------------------------------------------------------
template <typename Real, int R>
__device__ __forceinline__ void diag_ops(const Op& op, V2<Real> (&v)[1 << R], uint64_t gl, const uint64_t (&hb)[5],
                                         const V2<Real>* coef, const PolyTables& poly) {
  const uint32_t creg = op.creg;
  switch (op.type) {
    case OP_NEG:
      if ((gl & op.mask) == op.mask) dispatch_neg<Real, R>(v, creg);
      break;
    case OP_CPHASE: {
      const bool thr = (gl & op.mask) == op.mask;
      const V2<Real> c = ld_coef<Real>(coef + op.coef);
#pragma unroll
      for (int r = 0; r < (1 << R); ++r)
        if (AB_ON(r)) v[r] = cmul<Real>(c, v[r]);
      break;
    }
    case OP_DIAG: {
      const bool thr = (gl & op.ctrl) == op.ctrl;
      const int nq = op.nq;
      uint32_t tidx = 0;  // table-index bits taken from thread-constant qubits
#pragma unroll
      for (int i = 0; i < 3; ++i)
        if (i < nq && !((op.dsrc >> i) & 1)) tidx |= (uint32_t)((gl >> op.q[i]) & 1) << (nq - 1 - i);
      const uint32_t s0 = op.q[3], s1 = op.q[4], s2 = op.q[5];
      const uint32_t d0 = (op.dsrc >> 0) & 1, d1 = (op.dsrc >> 1) & 1, d2 = (op.dsrc >> 2) & 1;
      const V2<Real>* tab = coef + op.coef;
#pragma unroll
      for (int r = 0; r < (1 << R); ++r) {
        if (!AB_ON(r)) continue;
        uint32_t idx = tidx;
        if (d0) idx |= ((r >> s0) & 1) << (nq - 1);
        if (d1) idx |= ((r >> s1) & 1) << (nq - 2);
        if (d2) idx |= ((r >> s2) & 1) << (nq - 3);
        v[r] = cmul<Real>(ld_coef<Real>(tab + idx), v[r]);
      }
      break;
    }
    case OP_POLY: {
#pragma unroll
      for (int r = 0; r < (1 << R); ++r) v[r] = apply_diag_op<Real>(op, v[r], gl | roff<R>(r, hb), coef, poly);
      break;
    }
  }
}

template <typename Real, int R>
__device__ __forceinline__ void dispatch_reg(const Op& op, V2<Real> (&v)[1 << R], const V2<Real>* m, bool thr) {
  const uint32_t creg = op.creg;
  const int J = op.a - 5;
  if (op.type == OP_X) {
    switch (J) {
      case 0: if constexpr (R > 0) reg_x<Real, R, 0>(v, thr, creg); break;
      case 1: if constexpr (R > 1) reg_x<Real, R, 1>(v, thr, creg); break;
      case 2: if constexpr (R > 2) reg_x<Real, R, 2>(v, thr, creg); break;
      case 3: if constexpr (R > 3) reg_x<Real, R, 3>(v, thr, creg); break;
      case 4: if constexpr (R > 4) reg_x<Real, R, 4>(v, thr, creg); break;
    }
    return;
  }
  switch (J) {
    case 0: if constexpr (R > 0) reg_1q<Real, R, 0>(v, m, thr, creg); break;
    case 1: if constexpr (R > 1) reg_1q<Real, R, 1>(v, m, thr, creg); break;
    case 2: if constexpr (R > 2) reg_1q<Real, R, 2>(v, m, thr, creg); break;
    case 3: if constexpr (R > 3) reg_1q<Real, R, 3>(v, m, thr, creg); break;
    case 4: if constexpr (R > 4) reg_1q<Real, R, 4>(v, m, thr, creg); break;
  }
}

// Two uncontrolled one-qubit gates on register bits j1 != j2 (in that order).
template <typename Real, int R>
__device__ __forceinline__ void dispatch_pair(int j1, int j2, V2<Real> (&v)[1 << R], const V2<Real>* m,
                                              const V2<Real>* u) {
#define AB_PR(a, b)                                                      \
  case (a)*8 + (b):                                                      \
    if constexpr (R > (a) && R > (b)) reg_1q_pair<Real, R, (a), (b)>(v, m, u); \
    break;
  switch (j1 * 8 + j2) {
    AB_PR(0, 1) AB_PR(0, 2) AB_PR(0, 3) AB_PR(0, 4) AB_PR(1, 0) AB_PR(1, 2) AB_PR(1, 3) AB_PR(1, 4)
    AB_PR(2, 0) AB_PR(2, 1) AB_PR(2, 3) AB_PR(2, 4) AB_PR(3, 0) AB_PR(3, 1) AB_PR(3, 2) AB_PR(3, 4)
    AB_PR(4, 0) AB_PR(4, 1) AB_PR(4, 2) AB_PR(4, 3)
  }
#undef AB_PR
}

template <typename Real, int R, int QB>
__device__ __forceinline__ void dispatch_2q(const Op& op, V2<Real> (&v)[1 << R], const V2<Real>* m, bool thr) {
  const uint32_t creg = op.creg;
  // quartets per coefficient load in the uncontrolled register-register case
  constexpr int kQB = QB > (1 << (R >= 2 ? R - 2 : 0)) ? (1 << (R >= 2 ? R - 2 : 0)) : QB;
  if (op.b < 5) {
    if (op.a < 5) {
      lane_2q<Real, R>(v, op.a, op.b, m, thr, creg);
      return;
    }
    switch (op.a - 5) {
      case 0: if constexpr (R > 0) regl_2q<Real, R, 0>(v, op.b, m, thr, creg); break;
      case 1: if constexpr (R > 1) regl_2q<Real, R, 1>(v, op.b, m, thr, creg); break;
      case 2: if constexpr (R > 2) regl_2q<Real, R, 2>(v, op.b, m, thr, creg); break;
      case 3: if constexpr (R > 3) regl_2q<Real, R, 3>(v, op.b, m, thr, creg); break;
      case 4: if constexpr (R > 4) regl_2q<Real, R, 4>(v, op.b, m, thr, creg); break;
    }
    return;
  }
#define AB_RR(a, b)                                                           \
  case (a)*8 + (b):                                                           \
    if constexpr (R > (a)) {                                                  \
      if (kQB > 1 && thr && creg == 0) reg_2q_blocked<Real, R, (a), (b), kQB>(v, m); \
      else reg_2q<Real, R, (a), (b)>(v, m, thr, creg);                        \
    }                                                                         \
    break;
  switch ((op.a - 5) * 8 + (op.b - 5)) {
    AB_RR(1, 0) AB_RR(2, 0) AB_RR(2, 1) AB_RR(3, 0) AB_RR(3, 1)
    AB_RR(3, 2) AB_RR(4, 0) AB_RR(4, 1) AB_RR(4, 2) AB_RR(4, 3)
  }
#undef AB_RR
}

// ---- the warp-tile pass -----------------------------------------------------
// OCC: the resident 128-thread blocks per SM the variant is compiled for
// (register budget 65536 / (128 * OCC)); more resident warps hide more
// latency, fewer registers per thread cost spills at large R.
template <typename Real, int R, int OCC>
__global__ void __launch_bounds__(128, OCC) tile_kernel(V2<Real>* __restrict__ amps, const TilePass p,
                                                        const Op* __restrict__ ops, const V2<Real>* __restrict__ coef,
                                                        const PolyTables poly) {
  constexpr int NR = 1 << R;
  // quartets of a 4x4 per coefficient load: what the register budget
  // (65536 / (128 * OCC), at most 255) leaves beside the tile's amplitudes
  // for QB x 4 outputs and a row of coefficients
  constexpr int kRegBudget = 65536 / (128 * OCC) > 255 ? 255 : 65536 / (128 * OCC);
  constexpr int kRegData = (1 << R) * 2 * (int)sizeof(Real) / 4;
  constexpr int kCplx = 2 * (int)sizeof(Real) / 4;  // registers per complex value
  constexpr int kQuartetBlock = kRegBudget - kRegData >= (16 + 4) * kCplx + 40   ? 4
                                : kRegBudget - kRegData >= (8 + 4) * kCplx + 56 ? 2
                                                                                 : 1;
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
    const bool thr = (gl & op.ctrl) == op.ctrl;
    switch (op.type) {
      case OP_1Q: {
        if (op.a < 5) {
          lane_1q<Real, R>(v, op.a, m, thr, op.creg);
          break;
        }
        // gate pairs need the coefficients of both gates and a quartet of
        // temporaries live: only in the variants whose register budget
        // (65536 / (128 * OCC), at most 255) leaves room for them beside the
        // tile's amplitudes
        constexpr int kBudget = 65536 / (128 * OCC) > 255 ? 255 : 65536 / (128 * OCC);
        constexpr int kData = (1 << R) * 2 * (int)sizeof(Real) / 4;
        constexpr bool kPairs = R >= 2 && kBudget - kData >= 96;
        if (kPairs && op.ctrl == 0 && op.creg == 0 && i + 1 < p.op_count) {
          const Op nx = ops[p.op_begin + i + 1];
          if (nx.type == OP_1Q && nx.a >= 5 && nx.a != op.a && nx.ctrl == 0 && nx.creg == 0) {
            dispatch_pair<Real, R>(op.a - 5, nx.a - 5, v, m, coef + nx.coef);
            ++i;
            break;
          }
        }
        dispatch_reg<Real, R>(op, v, m, thr);
        break;
      }
      case OP_X:
        if (op.a < 5) lane_x<Real, R>(v, op.a, thr, op.creg);
        else dispatch_reg<Real, R>(op, v, m, thr);
        break;
      case OP_2Q:
        dispatch_2q<Real, R, kQuartetBlock>(op, v, m, thr);
        break;
      default:
        diag_ops<Real, R>(op, v, gl, hb, coef, poly);
        break;
    }
  }

#pragma unroll
  for (int r = 0; r < NR; ++r) st_amp<Real>(amps + (gl | roff<R>(r, hb)), v[r]);
}

template <typename Real, int R, int OCC>
static cudaError_t launch_tile_t(void* amps, const TilePass& p, const Op* ops, const void* coef, PolyTables poly,
                                 cudaStream_t s) {
  const uint64_t warps = 1ull << (p.n - 5 - R);
  const uint32_t wpb = 4;
  const uint64_t blocks = (warps + wpb - 1) / wpb;
  tile_kernel<Real, R, OCC>
      <<<(unsigned)blocks, 32 * wpb, 0, s>>>((V2<Real>*)amps, p, ops, (const V2<Real>*)coef, poly);
  return cudaGetLastError();
}

template <typename Real, int R>
static cudaError_t launch_tile_occ(void* amps, const TilePass& p, const Op* ops, const void* coef, PolyTables poly,
                                   cudaStream_t s) {
  // default: FP32 tiles run best at 4 blocks per SM, FP64 at 2 (measured on
  // the n=30 depth-40 brickwall: FP32 R=5 occ 2/3/4 = 1.22/1.00/0.94 s, FP64
  // R=5 occ 2/3 = 1.57/1.63 s)
  const uint32_t occ = p.occupancy ? p.occupancy : (sizeof(Real) == 4 ? 4u : 2u);
  switch (occ) {
    case 3: return launch_tile_t<Real, R, 3>(amps, p, ops, coef, poly, s);
    case 4: return launch_tile_t<Real, R, 4>(amps, p, ops, coef, poly, s);
    default: return launch_tile_t<Real, R, 2>(amps, p, ops, coef, poly, s);
  }
}

cudaError_t launch_tile_pass(void* amps, int precision, const TilePass& p, const Op* ops, const void* coef,
                             PolyTables poly, int* /*dev_error: no waits in this kernel*/, int /*sm_count*/,
                             cudaStream_t s) {
  if (p.R < 1 || p.R > 5 || p.n < 5 + p.R) return cudaErrorInvalidValue;
  const bool f64 = precision == ALEPH_B200_F64;
  switch (p.R) {
#define AB_TILE_CASE(RR)                                                        \
  case RR:                                                                      \
    return f64 ? launch_tile_occ<double, RR>(amps, p, ops, coef, poly, s)       \
               : launch_tile_occ<float, RR>(amps, p, ops, coef, poly, s);
    AB_TILE_CASE(1)
    AB_TILE_CASE(2)
    AB_TILE_CASE(3)
    AB_TILE_CASE(4)
    AB_TILE_CASE(5)
#undef AB_TILE_CASE
  }
  return cudaErrorInvalidValue;
}

}  // namespace ab
