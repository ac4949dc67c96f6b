// sv_oracle.cpp — TEST INFRASTRUCTURE, not product code.
//
// CPU FP64 restatement of aleph's reference state-vector backend
// (`NaiveSvBackend`, crates/aleph-sv/src/backend.rs:14-233) on its raw,
// gate-by-gate path. It is the checker for the B200 engine: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load it.
//
// The reference is Rust and cannot be compiled in this environment (no Rust
// toolchain, crates.io dependencies not vendored), so this file restates its
// algorithms. Each function cites the reference code it follows. Complex
// arithmetic follows num-complex 0.4 (the reference's `Complex<f64>`):
//   (a*b).re = a.re*b.re - a.im*b.im, (a*b).im = a.re*b.im + a.im*b.re,
// and the build disables FMA contraction (-ffp-contract=off) so every
// operation rounds like the Rust code.
//
// Parallelism: std::thread workers over disjoint contiguous index ranges, like
// the reference's rayon `par_blocks` (crates/aleph-sv/src/kernels/mod.rs:160-182);
// every amplitude is computed independently, so results do not depend on the
// thread count (ORACLE_THREADS, default: all hardware threads).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <cstdlib>
#include <thread>

#include "../include/aleph_b200.h"

namespace {

int oracle_threads() {
  static int t = [] {
    const char* e = std::getenv("ORACLE_THREADS");
    int v = e ? std::atoi(e) : 0;
    if (v <= 0) v = (int)std::thread::hardware_concurrency();
    return v <= 0 ? 1 : v;
  }();
  return t;
}

// Runs body(i) for i in [0, len) on disjoint contiguous ranges.
template <typename F>
void par_for(int64_t len, F body) {
  int nt = oracle_threads();
  if (len < (1 << 14) || nt == 1) {
    for (int64_t i = 0; i < len; ++i) body(i);
    return;
  }
  std::vector<std::thread> ws;
  int64_t chunk = (len + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    int64_t b = t * chunk, e = std::min(len, b + chunk);
    if (b >= e) break;
    ws.emplace_back([=] {
      for (int64_t i = b; i < e; ++i) body(i);
    });
  }
  for (auto& w : ws) w.join();
}

struct C {
  double re, im;
};
inline C cmul(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C cadd(C a, C b) { return {a.re + b.re, a.im + b.im}; }
inline C csub(C a, C b) { return {a.re - b.re, a.im - b.im}; }
inline C cconj(C a) { return {a.re, -a.im}; }
inline C cneg(C a) { return {-a.re, -a.im}; }
inline double cnorm(C a) { return std::hypot(a.re, a.im); }  // num-complex `norm()`
inline double cnorm_sqr(C a) { return a.re * a.re + a.im * a.im; }

// AMPLITUDE_TOL, crates/aleph-core/src/lib.rs:53
constexpr double kAmplitudeTol = 1e-10;
// DEGENERATE_BRANCH_THRESHOLD, crates/aleph-sv/src/measure.rs:12
constexpr double kDegenerate = 1e-300;

struct Err {
  int status = ALEPH_B200_OK;
  aleph_b200_error_info info{};
};

thread_local Err g_err;

int fail(int status) {
  g_err.info.status = status;
  g_err.status = status;
  return status;
}
void set_kind(const char* k) {
  std::snprintf(g_err.info.kind, sizeof(g_err.info.kind), "%s", k);
}

// Gate::name, crates/aleph-core/src/gate/kinds.rs:156-186
const char* gate_name(uint32_t kind) {
  static const char* names[] = {"H",    "X",      "Y",       "Z",         "S",         "Sdg",       "T",
                                "Tdg",  "Rx",     "Ry",      "Rz",        "Phase",     "U3",        "Cnot",
                                "Cz",   "Swap",   "Iswap",   "IswapDg",   "CRx",       "CRy",       "CRz",
                                "Toffoli", "Ccz", "Unitary1q", "Unitary2q", "UnitaryKq", "Unitary1qDiag",
                                "Unitary2qDiag"};
  if (kind < 28) return names[kind];
  switch (kind) {
    case ALEPH_INSTR_MEASURE: return "measure";
    case ALEPH_INSTR_RESET: return "reset";
    case ALEPH_INSTR_BARRIER: return "barrier";
    case ALEPH_INSTR_DIAGONAL_PHASE: return "diagonal_phase";
    case ALEPH_INSTR_TILED_BLOCK: return "tiled_block";
  }
  return "unknown";
}

// Gate::arity, crates/aleph-core/src/gate/kinds.rs:110-152
int gate_arity(const aleph_b200_instr& g) {
  switch (g.kind) {
    case ALEPH_GATE_H: case ALEPH_GATE_X: case ALEPH_GATE_Y: case ALEPH_GATE_Z: case ALEPH_GATE_S:
    case ALEPH_GATE_SDG: case ALEPH_GATE_T: case ALEPH_GATE_TDG: case ALEPH_GATE_RX: case ALEPH_GATE_RY:
    case ALEPH_GATE_RZ: case ALEPH_GATE_PHASE: case ALEPH_GATE_U3: case ALEPH_GATE_UNITARY1Q:
    case ALEPH_GATE_UNITARY1QDIAG:
      return 1;
    case ALEPH_GATE_CNOT: case ALEPH_GATE_CZ: case ALEPH_GATE_SWAP: case ALEPH_GATE_ISWAP:
    case ALEPH_GATE_ISWAPDG: case ALEPH_GATE_CRX: case ALEPH_GATE_CRY: case ALEPH_GATE_CRZ:
    case ALEPH_GATE_UNITARY2Q: case ALEPH_GATE_UNITARY2QDIAG:
      return 2;
    case ALEPH_GATE_TOFFOLI: case ALEPH_GATE_CCZ:
      return 3;
    case ALEPH_GATE_UNITARYKQ:
      return (int)g.aux;
  }
  return -1;
}

// Gate::matrix, crates/aleph-core/src/gate/kinds.rs:213-400. Returns dim (2/4/8)
// or 0 on error (g_err set).
int gate_matrix(const aleph_b200_instr& g, const double* pool, uint64_t pool_len, C m[8][8]) {
  const C zero{0.0, 0.0}, one{1.0, 0.0};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) m[i][j] = zero;
  auto concrete = [&](double v) -> bool {
    if (!std::isfinite(v)) {
      set_kind(gate_name(g.kind));
      fail(ALEPH_B200_NON_FINITE_PARAM);
      return false;
    }
    return true;
  };
  const double frac_1_sqrt_2 = 0.70710678118654752440;  // std::f64::consts::FRAC_1_SQRT_2
  const double frac_pi_4 = 0.78539816339744830962;      // std::f64::consts::FRAC_PI_4
  auto pool_at = [&](uint64_t idx) -> C { return C{pool[2 * idx], pool[2 * idx + 1]}; };
  auto need_pool = [&](uint64_t len) -> bool {
    if (!pool || g.data_len != len || g.data_offset + len > pool_len) {
      fail(ALEPH_B200_INVALID_ARGUMENT);
      return false;
    }
    return true;
  };
  switch (g.kind) {
    case ALEPH_GATE_H: {
      C s{frac_1_sqrt_2, 0.0};
      m[0][0] = s; m[0][1] = s; m[1][0] = s; m[1][1] = cneg(s);
      return 2;
    }
    case ALEPH_GATE_X: m[0][1] = one; m[1][0] = one; return 2;
    case ALEPH_GATE_Y: m[0][1] = C{0.0, -1.0}; m[1][0] = C{0.0, 1.0}; return 2;
    case ALEPH_GATE_Z: m[0][0] = one; m[1][1] = cneg(one); return 2;
    case ALEPH_GATE_S: m[0][0] = one; m[1][1] = C{0.0, 1.0}; return 2;
    case ALEPH_GATE_SDG: m[0][0] = one; m[1][1] = C{0.0, -1.0}; return 2;
    case ALEPH_GATE_T: m[0][0] = one; m[1][1] = C{std::cos(frac_pi_4), std::sin(frac_pi_4)}; return 2;
    case ALEPH_GATE_TDG: m[0][0] = one; m[1][1] = C{std::cos(frac_pi_4), -std::sin(frac_pi_4)}; return 2;
    case ALEPH_GATE_RX: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      C c{std::cos(t / 2.0), 0.0}, nis{0.0, -std::sin(t / 2.0)};
      m[0][0] = c; m[0][1] = nis; m[1][0] = nis; m[1][1] = c;
      return 2;
    }
    case ALEPH_GATE_RY: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      C c{std::cos(t / 2.0), 0.0}, s{std::sin(t / 2.0), 0.0};
      m[0][0] = c; m[0][1] = cneg(s); m[1][0] = s; m[1][1] = c;
      return 2;
    }
    case ALEPH_GATE_RZ: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      m[0][0] = C{std::cos(t / 2.0), -std::sin(t / 2.0)};
      m[1][1] = C{std::cos(t / 2.0), std::sin(t / 2.0)};
      return 2;
    }
    case ALEPH_GATE_PHASE: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      m[0][0] = one; m[1][1] = C{std::cos(t), std::sin(t)};
      return 2;
    }
    case ALEPH_GATE_U3: {
      for (int i = 0; i < 3; ++i)
        if (!concrete(g.params[i])) return 0;
      double t = g.params[0], f = g.params[1], l = g.params[2];
      C c{std::cos(t / 2.0), 0.0}, s{std::sin(t / 2.0), 0.0};
      C e_l{std::cos(l), std::sin(l)}, e_f{std::cos(f), std::sin(f)}, e_fl{std::cos(f + l), std::sin(f + l)};
      m[0][0] = c; m[0][1] = cneg(cmul(e_l, s)); m[1][0] = cmul(e_f, s); m[1][1] = cmul(e_fl, c);
      return 2;
    }
    case ALEPH_GATE_CNOT:
      m[0][0] = one; m[1][1] = one; m[2][3] = one; m[3][2] = one; return 4;
    case ALEPH_GATE_CZ:
      m[0][0] = one; m[1][1] = one; m[2][2] = one; m[3][3] = cneg(one); return 4;
    case ALEPH_GATE_SWAP:
      m[0][0] = one; m[1][2] = one; m[2][1] = one; m[3][3] = one; return 4;
    case ALEPH_GATE_ISWAP:
      m[0][0] = one; m[1][2] = C{0.0, 1.0}; m[2][1] = C{0.0, 1.0}; m[3][3] = one; return 4;
    case ALEPH_GATE_ISWAPDG:
      m[0][0] = one; m[1][2] = C{0.0, -1.0}; m[2][1] = C{0.0, -1.0}; m[3][3] = one; return 4;
    case ALEPH_GATE_CRX: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      C c{std::cos(t / 2.0), 0.0}, nis{0.0, -std::sin(t / 2.0)};
      m[0][0] = one; m[1][1] = one; m[2][2] = c; m[2][3] = nis; m[3][2] = nis; m[3][3] = c;
      return 4;
    }
    case ALEPH_GATE_CRY: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      C c{std::cos(t / 2.0), 0.0}, s{std::sin(t / 2.0), 0.0};
      m[0][0] = one; m[1][1] = one; m[2][2] = c; m[2][3] = cneg(s); m[3][2] = s; m[3][3] = c;
      return 4;
    }
    case ALEPH_GATE_CRZ: {
      if (!concrete(g.params[0])) return 0;
      double t = g.params[0];
      m[0][0] = one; m[1][1] = one;
      m[2][2] = C{std::cos(t / 2.0), -std::sin(t / 2.0)};
      m[3][3] = C{std::cos(t / 2.0), std::sin(t / 2.0)};
      return 4;
    }
    case ALEPH_GATE_TOFFOLI:
      for (int i = 0; i < 6; ++i) m[i][i] = one;
      m[6][7] = one; m[7][6] = one;
      return 8;
    case ALEPH_GATE_CCZ:
      for (int i = 0; i < 7; ++i) m[i][i] = one;
      m[7][7] = cneg(one);
      return 8;
    case ALEPH_GATE_UNITARY1Q:
      if (!need_pool(4)) return 0;
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) m[i][j] = pool_at(g.data_offset + 2 * i + j);
      return 2;
    case ALEPH_GATE_UNITARY2Q:
      if (!need_pool(16)) return 0;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m[i][j] = pool_at(g.data_offset + 4 * i + j);
      return 4;
    case ALEPH_GATE_UNITARY1QDIAG:
      if (!need_pool(2)) return 0;
      m[0][0] = pool_at(g.data_offset);
      m[1][1] = pool_at(g.data_offset + 1);
      return 2;
    case ALEPH_GATE_UNITARY2QDIAG:
      if (!need_pool(4)) return 0;
      for (int i = 0; i < 4; ++i) m[i][i] = pool_at(g.data_offset + i);
      return 4;
  }
  set_kind(gate_name(g.kind));
  fail(ALEPH_B200_UNSUPPORTED_GATE);
  return 0;
}

// unitarity_deviation, crates/aleph-sv/src/validation.rs:25-51
double unitarity_deviation(C m[8][8], int dim) {
  double worst = 0.0;
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) {
      C acc{0.0, 0.0};
      for (int c = 0; c < dim; ++c) acc = cadd(acc, cmul(m[i][c], cconj(m[j][c])));
      double dev = cnorm(csub(acc, C{i == j ? 1.0 : 0.0, 0.0}));
      if (std::isnan(dev)) return NAN;
      if (dev > worst) worst = dev;
    }
  return worst;
}

// validate_unitary_kq, crates/aleph-sv/src/validation.rs:113-155
int validate_unitary_kq(uint32_t k, const C* data, uint64_t len, uint32_t ncontrols) {
  if (k < 2 || k > 5) {
    set_kind("UnitaryKq width must be between 2 and 5");
    return fail(ALEPH_B200_INVALID_STATE);
  }
  if (ncontrols != 0) {
    set_kind("controlled UnitaryKq");
    return fail(ALEPH_B200_UNSUPPORTED_GATE);
  }
  uint64_t w = 1ull << k;
  if (len != w * w) {
    set_kind("UnitaryKq matrix length does not match width");
    return fail(ALEPH_B200_INVALID_STATE);
  }
  for (uint64_t i = 0; i < len; ++i)
    if (!std::isfinite(data[i].re) || !std::isfinite(data[i].im)) {
      set_kind("UnitaryKq");
      return fail(ALEPH_B200_NON_FINITE_PARAM);
    }
  double dev2 = 0.0;
  for (uint64_t i = 0; i < w; ++i)
    for (uint64_t j = 0; j <= i; ++j) {
      C sum{0.0, 0.0};
      for (uint64_t c = 0; c < w; ++c) sum = cadd(sum, cmul(data[i * w + c], cconj(data[j * w + c])));
      double e = cnorm_sqr(csub(sum, C{i == j ? 1.0 : 0.0, 0.0}));
      if (!std::isfinite(e)) {
        g_err.info.value = e;
        return fail(ALEPH_B200_NON_UNITARY_MATRIX);
      }
      dev2 = std::max(dev2, e);
    }
  if (dev2 > kAmplitudeTol * kAmplitudeTol) {
    g_err.info.value = std::sqrt(dev2);
    return fail(ALEPH_B200_NON_UNITARY_MATRIX);
  }
  return ALEPH_B200_OK;
}

// Dense k-target kernel with generic controls. Restates the scalar kernels
// apply_1q (crates/aleph-sv/src/kernels/aos.rs:192-223), apply_2q_dense_scalar
// (aos.rs:1335-1394), apply_3q_generic (aos.rs:3753-3832) and
// apply_kq_scalar_aos (crates/aleph-sv/src/kernels/unitary_kq.rs:127-166):
// operand order is MSB-first (matrix bit p <-> qubit targets[k-1-p]); each
// output row is the left-to-right sum of m[r][c] * v[c].
void apply_dense(C* amps, uint32_t n, const uint32_t* targets, int k, const C* m /* dim*dim */,
                 const uint32_t* controls, uint32_t nc) {
  const uint64_t dim = 1ull << k;
  uint64_t offsets[32];
  for (uint64_t r = 0; r < dim; ++r) {
    uint64_t off = 0;
    for (int p = 0; p < k; ++p)
      if ((r >> p) & 1) off |= 1ull << targets[k - 1 - p];
    offsets[r] = off;
  }
  uint64_t tmask = 0, cmask = 0;
  for (int i = 0; i < k; ++i) tmask |= 1ull << targets[i];
  for (uint32_t i = 0; i < nc; ++i) cmask |= 1ull << controls[i];
  const int64_t len = (int64_t)1 << n;
  par_for(len, [&](int64_t i) {
    uint64_t base = (uint64_t)i;
    if ((base & tmask) != 0 || (base & cmask) != cmask) return;
    C v[32];
    for (uint64_t c = 0; c < dim; ++c) v[c] = amps[base | offsets[c]];
    for (uint64_t r = 0; r < dim; ++r) {
      C acc{0.0, 0.0};
      for (uint64_t c = 0; c < dim; ++c) acc = cadd(acc, cmul(m[r * dim + c], v[c]));
      amps[base | offsets[r]] = acc;
    }
  });
}

// phase_at + apply_diagonal_phase_scalar_aos,
// crates/aleph-sv/src/kernels/diagonal_phase.rs:26-41,74-97
void apply_diag_phase(C* amps, uint32_t n, const aleph_b200_phase_term* terms, uint64_t nt, const uint64_t* conds) {
  const int64_t len = (int64_t)1 << n;
  par_for(len, [&](int64_t i) {
    uint64_t x = (uint64_t)i;
    double phi = 0.0;
    for (uint64_t t = 0; t < nt; ++t) {
      bool all = true;
      for (uint32_t c = 0; c < terms[t].cond_count; ++c)
        if ((__builtin_popcountll(conds[terms[t].cond_offset + c] & x) & 1) == 0) {
          all = false;
          break;
        }
      if (all) phi += terms[t].angle;
    }
    double s = std::sin(phi), co = std::cos(phi);
    C a = amps[i];
    amps[i] = C{a.re * co - a.im * s, a.re * s + a.im * co};
  });
}

// validate_norm, crates/aleph-sv/src/sampling.rs:36-57; validate_state,
// crates/aleph-sv/src/measure.rs:23-33. Sequential left-to-right sum.
int validate_state(const C* amps, uint32_t n, std::vector<double>* probs, double* total_out) {
  const uint64_t len = 1ull << n;
  double total = 0.0;
  if (probs) probs->resize(len);
  for (uint64_t i = 0; i < len; ++i) {
    double p = cnorm_sqr(amps[i]);
    if (!std::isfinite(p)) {
      set_kind("non-finite amplitude norm\xc2\xb2");
      return fail(ALEPH_B200_INVALID_STATE);
    }
    total += p;
    if (probs) (*probs)[i] = p;
  }
  double tol = std::sqrt((double)len) * kAmplitudeTol;
  if (!std::isfinite(total) || std::fabs(total - 1.0) > tol) {
    set_kind("state norm\xc2\xb2 deviates from 1 beyond drift budget");
    return fail(ALEPH_B200_INVALID_STATE);
  }
  if (total_out) *total_out = total;
  return ALEPH_B200_OK;
}

int check_qubits(const uint32_t* q, uint32_t k, uint32_t n) {
  for (uint32_t i = 0; i < k; ++i) {
    if (q[i] >= n) {
      g_err.info.qubit = q[i];
      g_err.info.num_qubits = n;
      return fail(ALEPH_B200_QUBIT_OUT_OF_RANGE);
    }
    for (uint32_t j = 0; j < i; ++j)
      if (q[j] == q[i]) {
        g_err.info.qubit = q[i];
        return fail(ALEPH_B200_DUPLICATE_QUBIT);
      }
  }
  return ALEPH_B200_OK;
}

}  // namespace

namespace {
int apply_gate_impl(double* amps_d, uint32_t n, const aleph_b200_instr* g, const double* pool, uint64_t pool_len,
                    bool tiled);
}

extern "C" {

// Reset the thread-local error before each call.
static void clear_err() { g_err = Err{}; }

int orc_last_error(aleph_b200_error_info* out) {
  if (out) *out = g_err.info;
  return g_err.status;
}

// NaiveSvBackend::allocate, crates/aleph-sv/src/backend.rs:61-72 (caller owns `amps`, 2*2^n doubles).
int orc_init(double* amps, uint32_t n) {
  clear_err();
  const uint64_t len = 1ull << n;
  std::memset(amps, 0, sizeof(double) * 2 * len);
  amps[0] = 1.0;
  return ALEPH_B200_OK;
}

// NaiveSvBackend::apply_gate, crates/aleph-sv/src/backend.rs:74-152: arity,
// bounds and duplicates (qubits then controls), UnitaryKq validation, matrix
// materialisation, unitarity check (deviation > 1e-10 rejects), dispatch.
int orc_apply_gate(double* amps_d, uint32_t n, const aleph_b200_instr* g, const double* pool, uint64_t pool_len) {
  return apply_gate_impl(amps_d, n, g, pool, pool_len, false);
}

// One gate of a TiledBlock: NaiveSvBackend::apply_tiled_block and
// dispatch_tile_kernel (crates/aleph-sv/src/backend.rs:173-208,265-299) take
// the gate's fixed-size matrix (Gate::matrix errors as for apply_gate;
// UnitaryKq has none: UnsupportedGate), route 2x2 and 4x4 to the tile
// kernels, reject 8x8 as UnsupportedGate, and make no unitarity check. The
// tile-by-tile order gives the same amplitudes as applying the gates to the
// whole state one after another (backend.rs:420-457), which is done here.
int orc_apply_tiled_gate(double* amps_d, uint32_t n, const aleph_b200_instr* g, const double* pool,
                         uint64_t pool_len) {
  return apply_gate_impl(amps_d, n, g, pool, pool_len, true);
}
}  // extern "C"

namespace {
int apply_gate_impl(double* amps_d, uint32_t n, const aleph_b200_instr* g, const double* pool, uint64_t pool_len,
                    bool tiled) {
  clear_err();
  C* amps = reinterpret_cast<C*>(amps_d);
  int expected = gate_arity(*g);
  if (expected < 0) {
    set_kind(gate_name(g->kind));
    return fail(ALEPH_B200_UNSUPPORTED_GATE);
  }
  if ((uint32_t)expected != g->num_qubits) {
    set_kind(gate_name(g->kind));
    g_err.info.expected = (uint32_t)expected;
    g_err.info.got = g->num_qubits;
    return fail(ALEPH_B200_ARITY_MISMATCH);
  }
  if (g->num_qubits > 8 || g->num_controls > 8) return fail(ALEPH_B200_INVALID_ARGUMENT);
  uint32_t all[16];
  uint32_t na = 0;
  for (uint32_t i = 0; i < g->num_qubits; ++i) all[na++] = g->qubits[i];
  for (uint32_t i = 0; i < g->num_controls; ++i) all[na++] = g->controls[i];
  if (int s = check_qubits(all, na, n)) return s;
  if (tiled && g->kind == ALEPH_GATE_UNITARYKQ) {
    set_kind(gate_name(g->kind));
    return fail(ALEPH_B200_UNSUPPORTED_GATE);
  }
  if (g->kind == ALEPH_GATE_UNITARYKQ) {
    uint32_t k = g->aux;
    if (!pool || g->data_offset + g->data_len > pool_len) return fail(ALEPH_B200_INVALID_ARGUMENT);
    const C* data = reinterpret_cast<const C*>(pool) + g->data_offset;
    if (int s = validate_unitary_kq(k, data, g->data_len, g->num_controls)) return s;
    apply_dense(amps, n, g->qubits, (int)k, data, nullptr, 0);
    return ALEPH_B200_OK;
  }
  C m[8][8];
  int dim = gate_matrix(*g, pool, pool_len, m);
  if (dim == 0) return g_err.status;
  if (tiled && dim > 4) {
    set_kind(gate_name(g->kind));
    return fail(ALEPH_B200_UNSUPPORTED_GATE);
  }
  if (!tiled) {
    double dev = unitarity_deviation(m, dim);
    if (!std::isfinite(dev) || dev > kAmplitudeTol) {
      g_err.info.value = dev;
      return fail(ALEPH_B200_NON_UNITARY_MATRIX);
    }
  }
  C flat[64];
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) flat[i * dim + j] = m[i][j];
  int k = dim == 2 ? 1 : dim == 4 ? 2 : 3;
  apply_dense(amps, n, g->qubits, k, flat, g->controls, g->num_controls);
  return ALEPH_B200_OK;
}
}  // namespace

extern "C" {

// Gate matrix (for tests of the host-side matrix builder). Writes dim*dim complex.
int orc_gate_matrix(const aleph_b200_instr* g, const double* pool, uint64_t pool_len, double* out, int* dim_out) {
  clear_err();
  C m[8][8];
  int dim = gate_matrix(*g, pool, pool_len, m);
  if (dim == 0) return g_err.status;
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) {
      out[2 * (i * dim + j)] = m[i][j].re;
      out[2 * (i * dim + j) + 1] = m[i][j].im;
    }
  *dim_out = dim;
  return ALEPH_B200_OK;
}

int orc_apply_diagonal_phase(double* amps, uint32_t n, const aleph_b200_phase_term* terms, uint64_t nt,
                             const uint64_t* conds, uint64_t nconds) {
  clear_err();
  for (uint64_t t = 0; t < nt; ++t)
    if ((uint64_t)terms[t].cond_offset + terms[t].cond_count > nconds) return fail(ALEPH_B200_INVALID_ARGUMENT);
  apply_diag_phase(reinterpret_cast<C*>(amps), n, terms, nt, conds);
  return ALEPH_B200_OK;
}

// bit_permute_buf, crates/aleph-core/src/perm.rs:25-40 (out-of-place gather).
int orc_unpermute(double* amps_d, uint32_t n, const uint32_t* perm) {
  clear_err();
  C* amps = reinterpret_cast<C*>(amps_d);
  const int64_t len = (int64_t)1 << n;
  std::vector<C> out((size_t)len);
  par_for(len, [&](int64_t i) {
    uint64_t j = 0;
    for (uint32_t lq = 0; lq < n; ++lq)
      if (((uint64_t)i >> lq) & 1) j |= 1ull << perm[lq];
    out[(size_t)i] = amps[j];
  });
  std::memcpy(amps, out.data(), sizeof(C) * (size_t)len);
  return ALEPH_B200_OK;
}

// measure_impl, crates/aleph-sv/src/measure.rs:41-102. `u` replaces
// rng.gen::<f64>() and is used only when both branches are non-degenerate.
int orc_measure(double* amps_d, uint32_t n, uint32_t qubit, double u, int* outcome_out, int* consumed) {
  clear_err();
  C* amps = reinterpret_cast<C*>(amps_d);
  *consumed = 0;
  if (qubit >= n) {
    g_err.info.qubit = qubit;
    g_err.info.num_qubits = n;
    return fail(ALEPH_B200_QUBIT_OUT_OF_RANGE);
  }
  std::vector<double> probs;
  if (int s = validate_state(amps, n, &probs, nullptr)) return s;
  const uint64_t qb = 1ull << qubit;
  double p0 = 0.0, p1 = 0.0;
  for (uint64_t i = 0; i < probs.size(); ++i) {
    if (i & qb) p1 += probs[i];
    else p0 += probs[i];
  }
  p0 = std::min(std::max(p0, 0.0), 1.0);
  p1 = std::min(std::max(p1, 0.0), 1.0);
  bool one_degen = p1 < kDegenerate, zero_degen = p0 < kDegenerate;
  bool outcome;
  double p;
  if (zero_degen && one_degen) {
    g_err.info.qubit = qubit;
    g_err.info.value = std::max(p1, p0);
    return fail(ALEPH_B200_DEGENERATE_MEASUREMENT);
  } else if (zero_degen) {
    outcome = true;
    p = p1;
  } else if (one_degen) {
    outcome = false;
    p = p0;
  } else {
    outcome = u < p1;
    *consumed = 1;
    p = outcome ? p1 : p0;
  }
  const double norm = std::sqrt(p);
  const int64_t len = (int64_t)1 << n;
  par_for(len, [&](int64_t i) {
    bool bit = ((uint64_t)i & qb) != 0;
    if (bit == outcome) {
      // num-complex `a /= Complex::new(norm, 0.0)`: (a * conj(b)) / |b|^2
      C a = amps[i];
      double d = norm * norm + 0.0 * 0.0;
      amps[i] = C{(a.re * norm + a.im * 0.0) / d, (a.im * norm - a.re * 0.0) / d};
    } else {
      amps[i] = C{0.0, 0.0};
    }
  });
  *outcome_out = outcome ? 1 : 0;
  return ALEPH_B200_OK;
}

// cumulative_index, crates/aleph-sv/src/sampling.rs:59-81.
static int cumulative_index(const std::vector<double>& probs, double target, uint64_t* out) {
  double cum = 0.0;
  int64_t last_pos = -1;
  for (uint64_t i = 0; i < probs.size(); ++i) {
    double p = probs[i];
    if (p > 0.0) {
      last_pos = (int64_t)i;
      cum += p;
      if (target < cum) {
        *out = i;
        return ALEPH_B200_OK;
      }
    }
  }
  if (last_pos < 0) {
    set_kind("state has no positive probability");
    return fail(ALEPH_B200_INVALID_STATE);
  }
  *out = (uint64_t)last_pos;
  return ALEPH_B200_OK;
}

// Inverse-CDF sampling, one double per shot: draw_cumulative
// (crates/aleph-sv/src/sampling.rs:83-91) applied per shot after one
// validate_norm (the reference's shots <= 1 path, measure.rs:128-148).
int orc_sample_cumulative(const double* amps_d, uint32_t n, uint32_t shots, const double* uniforms, uint64_t* out) {
  clear_err();
  const C* amps = reinterpret_cast<const C*>(amps_d);
  std::vector<double> probs;
  double total = 0.0;
  if (int s = validate_state(amps, n, &probs, &total)) return s;
  for (uint32_t s = 0; s < shots; ++s)
    if (int st = cumulative_index(probs, uniforms[s] * total, &out[s])) return st;
  return ALEPH_B200_OK;
}

// AliasTable::build (Vose 1991, Algorithm 3), crates/aleph-sv/src/sampling.rs:104-167.
static void alias_build(const std::vector<double>& p, std::vector<double>& prob, std::vector<uint32_t>& alias) {
  const size_t n = p.size();
  prob.assign(n, 0.0);
  alias.assign(n, 0);
  if (n == 1) {
    prob[0] = 1.0;
    return;
  }
  const double nf = (double)n;
  std::vector<double> scaled(n);
  for (size_t i = 0; i < n; ++i) scaled[i] = nf * p[i];
  std::vector<uint32_t> small, large;
  small.reserve(n);
  large.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    if (scaled[i] < 1.0) small.push_back((uint32_t)i);
    else large.push_back((uint32_t)i);
  }
  while (!small.empty() && !large.empty()) {
    uint32_t s = small.back();
    small.pop_back();
    uint32_t l = large.back();
    large.pop_back();
    prob[s] = scaled[s];
    alias[s] = l;
    double new_l = (scaled[l] + scaled[s]) - 1.0;
    scaled[l] = new_l;
    if (new_l < 1.0) small.push_back(l);
    else large.push_back(l);
  }
  for (uint32_t i : large) {
    prob[i] = 1.0;
    alias[i] = i;
  }
  for (uint32_t i : small) {
    prob[i] = 1.0;
    alias[i] = i;
  }
}

// Alias sampling, one u64 word per shot: AliasTable::draw,
// crates/aleph-sv/src/sampling.rs:179-197 (the reference's shots >= 2 path,
// measure.rs:109-124): index = (word >> 32) & (N-1), u = (u32)word / 2^32.
int orc_sample_alias(const double* amps_d, uint32_t n, uint32_t shots, const uint64_t* words, uint64_t* out) {
  clear_err();
  const C* amps = reinterpret_cast<const C*>(amps_d);
  std::vector<double> probs;
  if (int s = validate_state(amps, n, &probs, nullptr)) return s;
  std::vector<double> prob;
  std::vector<uint32_t> alias;
  alias_build(probs, prob, alias);
  const uint64_t mask = probs.size() - 1;
  for (uint32_t s = 0; s < shots; ++s) {
    uint64_t bits = words[s];
    uint64_t i = (bits >> 32) & mask;
    double u = (double)(uint32_t)bits * (1.0 / 4294967296.0);
    out[s] = u < prob[i] ? i : alias[i];
  }
  return ALEPH_B200_OK;
}

// Exposes the alias table itself (for tests of the device-side build).
int orc_alias_table(const double* probs, uint64_t len, double* prob_out, uint32_t* alias_out) {
  clear_err();
  std::vector<double> p(probs, probs + len), prob;
  std::vector<uint32_t> alias;
  alias_build(p, prob, alias);
  std::memcpy(prob_out, prob.data(), sizeof(double) * len);
  std::memcpy(alias_out, alias.data(), sizeof(uint32_t) * len);
  return ALEPH_B200_OK;
}

// expectation_value_impl, crates/aleph-sv/src/measure.rs:155-233.
int orc_expectation(const double* amps_d, uint32_t n, const uint32_t* qubits, const uint8_t* paulis, uint32_t nt,
                    double coefficient, double* out) {
  clear_err();
  const C* amps = reinterpret_cast<const C*>(amps_d);
  std::vector<double> probs;
  if (int s = validate_state(amps, n, &probs, nullptr)) return s;
  if (!std::isfinite(coefficient)) {
    set_kind("non-finite coefficient");
    return fail(ALEPH_B200_INVALID_PAULI_STRING);
  }
  if (int s = check_qubits(qubits, nt, n)) return s;
  uint64_t zmask = 0;
  bool all_z = true;
  for (uint32_t t = 0; t < nt; ++t) {
    if (paulis[t] == ALEPH_PAULI_Z) zmask |= 1ull << qubits[t];
    else if (paulis[t] == ALEPH_PAULI_X || paulis[t] == ALEPH_PAULI_Y) all_z = false;
    else if (paulis[t] != ALEPH_PAULI_I) return fail(ALEPH_B200_INVALID_ARGUMENT);
  }
  if (all_z) {
    // expectation_z_diag, measure.rs:289-300
    double acc = 0.0;
    for (uint64_t i = 0; i < probs.size(); ++i) {
      double sign = (__builtin_popcountll(i & zmask) & 1) == 0 ? 1.0 : -1.0;
      acc += sign * probs[i];
    }
    *out = coefficient * acc;
    return ALEPH_B200_OK;
  }
  const uint64_t len = 1ull << n;
  std::vector<C> tmp(amps, amps + len);
  for (uint32_t t = 0; t < nt; ++t) {
    C m[4];
    const C z{0.0, 0.0}, o{1.0, 0.0};
    switch (paulis[t]) {  // Pauli::matrix, crates/aleph-core/src/pauli.rs:21-33
      case ALEPH_PAULI_I: continue;
      case ALEPH_PAULI_X: m[0] = z; m[1] = o; m[2] = o; m[3] = z; break;
      case ALEPH_PAULI_Y: m[0] = z; m[1] = C{0.0, -1.0}; m[2] = C{0.0, 1.0}; m[3] = z; break;
      default: m[0] = o; m[1] = z; m[2] = z; m[3] = C{-1.0, 0.0}; break;
    }
    apply_dense(tmp.data(), n, &qubits[t], 1, m, nullptr, 0);
  }
  C acc{0.0, 0.0};
  for (uint64_t i = 0; i < len; ++i) acc = cadd(acc, cmul(cconj(amps[i]), tmp[i]));
  *out = coefficient * acc.re;
  return ALEPH_B200_OK;
}

// probabilities_impl, crates/aleph-sv/src/measure.rs:239-273 (qubits[0] = LSB).
int orc_probabilities(const double* amps_d, uint32_t n, const uint32_t* qubits, uint32_t k, double* out) {
  clear_err();
  const C* amps = reinterpret_cast<const C*>(amps_d);
  std::vector<double> probs;
  if (int s = validate_state(amps, n, &probs, nullptr)) return s;
  if (int s = check_qubits(qubits, k, n)) return s;
  if (k == 0) {
    out[0] = 1.0;
    return ALEPH_B200_OK;
  }
  const uint64_t od = 1ull << k;
  for (uint64_t o = 0; o < od; ++o) out[o] = 0.0;
  for (uint64_t i = 0; i < probs.size(); ++i) {
    uint64_t kk = 0;
    for (uint32_t pos = 0; pos < k; ++pos)
      if ((i >> qubits[pos]) & 1) kk |= 1ull << pos;
    out[kk] += probs[i];
  }
  return ALEPH_B200_OK;
}

// Sequential FP64 sum of |a|^2 (the validate_norm total).
int orc_norm_sqr(const double* amps_d, uint32_t n, double* out) {
  clear_err();
  const C* amps = reinterpret_cast<const C*>(amps_d);
  double total = 0.0;
  for (uint64_t i = 0; i < (1ull << n); ++i) total += cnorm_sqr(amps[i]);
  *out = total;
  return ALEPH_B200_OK;
}

// run_with_outcomes, crates/aleph-backend/src/lib.rs:211-245, over the flat
// instruction stream. Measurements take one uniform from `uniforms` each time
// both branches are non-degenerate. The gates of a TILED_BLOCK record follow
// it and go through orc_apply_tiled_gate (NaiveSvBackend::apply_tiled_block,
// crates/aleph-sv/src/backend.rs:173-299).
int orc_run_stream(double* amps, uint32_t n, const aleph_b200_instr* instrs, uint64_t count,
                   const aleph_b200_pools* pools, const double* uniforms, uint64_t n_uniforms, uint8_t* outcomes,
                   uint64_t outcomes_cap, uint64_t* n_outcomes, uint64_t* failed_at) {
  clear_err();
  uint64_t used = 0, nout = 0, tiled_left = 0;
  *failed_at = UINT64_MAX;
  for (uint64_t i = 0; i < count; ++i) {
    const aleph_b200_instr& g = instrs[i];
    int s = ALEPH_B200_OK;
    const bool tiled = tiled_left > 0;
    if (tiled) --tiled_left;
    if (tiled && g.kind >= 28) {
      clear_err();
      set_kind("tiled block member");
      s = fail(ALEPH_B200_INVALID_ARGUMENT);
    } else if (g.kind < 28) {
      s = apply_gate_impl(amps, n, &g, pools ? pools->matrix_pool : nullptr, pools ? pools->matrix_pool_len : 0,
                          tiled);
    } else if (g.kind == ALEPH_INSTR_MEASURE) {
      if (g.num_qubits != 1) {
        s = fail(ALEPH_B200_INVALID_ARGUMENT);
      } else {
        double u = used < n_uniforms ? uniforms[used] : NAN;
        int outcome = 0, consumed = 0;
        s = orc_measure(amps, n, g.qubits[0], u, &outcome, &consumed);
        if (s == ALEPH_B200_OK && consumed) {
          if (used >= n_uniforms) {
            set_kind("measure uniforms exhausted");
            s = fail(ALEPH_B200_INVALID_ARGUMENT);
          }
          ++used;
        }
        if (s == ALEPH_B200_OK) {
          if (nout < outcomes_cap) outcomes[nout] = (uint8_t)outcome;
          ++nout;
        }
      }
    } else if (g.kind == ALEPH_INSTR_RESET) {
      clear_err();
      set_kind("reset");
      s = fail(ALEPH_B200_UNSUPPORTED_INSTRUCTION);
    } else if (g.kind == ALEPH_INSTR_BARRIER) {
      s = ALEPH_B200_OK;
    } else if (g.kind == ALEPH_INSTR_TILED_BLOCK) {
      if (g.data_len > count - i - 1) {
        clear_err();
        set_kind("tiled block length");
        s = fail(ALEPH_B200_INVALID_ARGUMENT);
      }
      tiled_left = g.data_len;
    } else if (g.kind == ALEPH_INSTR_DIAGONAL_PHASE) {
      if (!pools || g.data_offset + g.data_len > pools->n_terms) s = fail(ALEPH_B200_INVALID_ARGUMENT);
      else
        s = orc_apply_diagonal_phase(amps, n, pools->terms + g.data_offset, g.data_len, pools->cond_pool,
                                     pools->n_conds);
    } else {
      clear_err();
      set_kind(gate_name(g.kind));
      s = fail(ALEPH_B200_UNSUPPORTED_INSTRUCTION);
    }
    if (s != ALEPH_B200_OK) {
      g_err.info.instruction = (uint32_t)i;
      *failed_at = i;
      *n_outcomes = nout;
      return s;
    }
  }
  *n_outcomes = nout;
  return ALEPH_B200_OK;
}

}  // extern "C"
