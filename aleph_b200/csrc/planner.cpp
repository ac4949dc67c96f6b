// planner.cpp — gate validation, lowering to device ops, and pass planning.
//
// Validation follows NaiveSvBackend::apply_gate (crates/aleph-sv/src/backend.rs:74-152)
// in the same order, with the same error variants: arity, then range and
// duplicates over qubits followed by controls, UnitaryKq validation
// (crates/aleph-sv/src/validation.rs:113-155), matrix materialisation
// (Gate::matrix, crates/aleph-core/src/gate/kinds.rs:213-400) and the
// unitarity check (validation.rs:25-51, AMPLITUDE_TOL = 1e-10).
//
// Planning: the gate list is cut into HBM passes. A warp-tile pass owns
// qubits 0..4 plus R "register" qubits; the planner walks the pending gates
// in order and takes every gate that (a) commutes past all gates it defers
// and (b) acts non-diagonally only on tile qubits — diagonal gates (CZ,
// phases, DiagonalPhase) and controls may sit on any qubit. This is the
// greedy open-block idea of FuseKq (crates/aleph-ir/src/passes/fuse_kq.rs:144-400)
// applied to cache tiles instead of matrices: no matrix is ever formed, the
// gates run in registers one after the other.

#include <algorithm>
#include <deque>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>

#include "engine.h"

namespace ab {

namespace {

struct Cx {
  double re, im;
};
inline Cx mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx add(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx sub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx conj(Cx a) { return {a.re, -a.im}; }
inline Cx neg(Cx a) { return {-a.re, -a.im}; }

constexpr double kTol = 1e-10;  // AMPLITUDE_TOL, crates/aleph-core/src/lib.rs:53

void set_kind(aleph_b200_error_info* e, const char* k) { std::snprintf(e->kind, sizeof(e->kind), "%s", k); }
int fail(aleph_b200_error_info* e, int s) {
  e->status = s;
  return s;
}

int arity(const aleph_b200_instr& g) {
  switch (g.kind) {
    case ALEPH_GATE_CNOT: case ALEPH_GATE_CZ: case ALEPH_GATE_SWAP: case ALEPH_GATE_ISWAP:
    case ALEPH_GATE_ISWAPDG: case ALEPH_GATE_CRX: case ALEPH_GATE_CRY: case ALEPH_GATE_CRZ:
    case ALEPH_GATE_UNITARY2Q: case ALEPH_GATE_UNITARY2QDIAG:
      return 2;
    case ALEPH_GATE_TOFFOLI: case ALEPH_GATE_CCZ:
      return 3;
    case ALEPH_GATE_UNITARYKQ:
      return (int)g.aux;
    default:
      return g.kind < 28 ? 1 : -1;
  }
}

// Gate::matrix (kinds.rs:213-400). Returns dim or 0 (error set).
int matrix_of(const aleph_b200_instr& g, const double* pool, uint64_t pool_len, Cx m[8][8],
              aleph_b200_error_info* e) {
  const Cx z{0, 0}, o{1, 0};
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) m[i][j] = z;
  for (int i = 0; i < 3; ++i) {
    const bool used = (g.kind >= ALEPH_GATE_RX && g.kind <= ALEPH_GATE_PHASE && i == 0) ||
                      (g.kind == ALEPH_GATE_U3) ||
                      ((g.kind == ALEPH_GATE_CRX || g.kind == ALEPH_GATE_CRY || g.kind == ALEPH_GATE_CRZ) && i == 0);
    if (used && !std::isfinite(g.params[i])) {
      set_kind(e, gate_name(g.kind));
      return fail(e, ALEPH_B200_NON_FINITE_PARAM), 0;
    }
  }
  const double s2 = 0.70710678118654752440, pi4 = 0.78539816339744830962;
  auto from_pool = [&](uint64_t len) -> const double* {
    if (!pool || g.data_len != len || g.data_offset + len > pool_len) {
      set_kind(e, "matrix pool");
      fail(e, ALEPH_B200_INVALID_ARGUMENT);
      return nullptr;
    }
    return pool + 2 * g.data_offset;
  };
  const double t = g.params[0];
  switch (g.kind) {
    case ALEPH_GATE_H: m[0][0] = m[0][1] = m[1][0] = Cx{s2, 0}; m[1][1] = Cx{-s2, 0}; return 2;
    case ALEPH_GATE_X: m[0][1] = m[1][0] = o; return 2;
    case ALEPH_GATE_Y: m[0][1] = Cx{0, -1}; m[1][0] = Cx{0, 1}; return 2;
    case ALEPH_GATE_Z: m[0][0] = o; m[1][1] = neg(o); return 2;
    case ALEPH_GATE_S: m[0][0] = o; m[1][1] = Cx{0, 1}; return 2;
    case ALEPH_GATE_SDG: m[0][0] = o; m[1][1] = Cx{0, -1}; return 2;
    case ALEPH_GATE_T: m[0][0] = o; m[1][1] = Cx{std::cos(pi4), std::sin(pi4)}; return 2;
    case ALEPH_GATE_TDG: m[0][0] = o; m[1][1] = Cx{std::cos(pi4), -std::sin(pi4)}; return 2;
    case ALEPH_GATE_RX:
      m[0][0] = m[1][1] = Cx{std::cos(t / 2), 0};
      m[0][1] = m[1][0] = Cx{0, -std::sin(t / 2)};
      return 2;
    case ALEPH_GATE_RY:
      m[0][0] = m[1][1] = Cx{std::cos(t / 2), 0};
      m[0][1] = Cx{-std::sin(t / 2), 0};
      m[1][0] = Cx{std::sin(t / 2), 0};
      return 2;
    case ALEPH_GATE_RZ:
      m[0][0] = Cx{std::cos(t / 2), -std::sin(t / 2)};
      m[1][1] = Cx{std::cos(t / 2), std::sin(t / 2)};
      return 2;
    case ALEPH_GATE_PHASE: m[0][0] = o; m[1][1] = Cx{std::cos(t), std::sin(t)}; return 2;
    case ALEPH_GATE_U3: {
      const double f = g.params[1], l = g.params[2];
      const Cx c{std::cos(t / 2), 0}, s{std::sin(t / 2), 0};
      m[0][0] = c;
      m[0][1] = neg(mul(Cx{std::cos(l), std::sin(l)}, s));
      m[1][0] = mul(Cx{std::cos(f), std::sin(f)}, s);
      m[1][1] = mul(Cx{std::cos(f + l), std::sin(f + l)}, c);
      return 2;
    }
    case ALEPH_GATE_CNOT: m[0][0] = m[1][1] = m[2][3] = m[3][2] = o; return 4;
    case ALEPH_GATE_CZ: m[0][0] = m[1][1] = m[2][2] = o; m[3][3] = neg(o); return 4;
    case ALEPH_GATE_SWAP: m[0][0] = m[1][2] = m[2][1] = m[3][3] = o; return 4;
    case ALEPH_GATE_ISWAP: m[0][0] = m[3][3] = o; m[1][2] = m[2][1] = Cx{0, 1}; return 4;
    case ALEPH_GATE_ISWAPDG: m[0][0] = m[3][3] = o; m[1][2] = m[2][1] = Cx{0, -1}; return 4;
    case ALEPH_GATE_CRX:
      m[0][0] = m[1][1] = o;
      m[2][2] = m[3][3] = Cx{std::cos(t / 2), 0};
      m[2][3] = m[3][2] = Cx{0, -std::sin(t / 2)};
      return 4;
    case ALEPH_GATE_CRY:
      m[0][0] = m[1][1] = o;
      m[2][2] = m[3][3] = Cx{std::cos(t / 2), 0};
      m[2][3] = Cx{-std::sin(t / 2), 0};
      m[3][2] = Cx{std::sin(t / 2), 0};
      return 4;
    case ALEPH_GATE_CRZ:
      m[0][0] = m[1][1] = o;
      m[2][2] = Cx{std::cos(t / 2), -std::sin(t / 2)};
      m[3][3] = Cx{std::cos(t / 2), std::sin(t / 2)};
      return 4;
    case ALEPH_GATE_TOFFOLI:
      for (int i = 0; i < 6; ++i) m[i][i] = o;
      m[6][7] = m[7][6] = o;
      return 8;
    case ALEPH_GATE_CCZ:
      for (int i = 0; i < 7; ++i) m[i][i] = o;
      m[7][7] = neg(o);
      return 8;
    case ALEPH_GATE_UNITARY1Q: {
      const double* p = from_pool(4);
      if (!p) return 0;
      for (int i = 0; i < 4; ++i) m[i / 2][i % 2] = Cx{p[2 * i], p[2 * i + 1]};
      return 2;
    }
    case ALEPH_GATE_UNITARY2Q: {
      const double* p = from_pool(16);
      if (!p) return 0;
      for (int i = 0; i < 16; ++i) m[i / 4][i % 4] = Cx{p[2 * i], p[2 * i + 1]};
      return 4;
    }
    case ALEPH_GATE_UNITARY1QDIAG: {
      const double* p = from_pool(2);
      if (!p) return 0;
      m[0][0] = Cx{p[0], p[1]};
      m[1][1] = Cx{p[2], p[3]};
      return 2;
    }
    case ALEPH_GATE_UNITARY2QDIAG: {
      const double* p = from_pool(4);
      if (!p) return 0;
      for (int i = 0; i < 4; ++i) m[i][i] = Cx{p[2 * i], p[2 * i + 1]};
      return 4;
    }
  }
  set_kind(e, gate_name(g.kind));
  fail(e, ALEPH_B200_UNSUPPORTED_GATE);
  return 0;
}

double unitarity_deviation(const Cx* m, int dim) {
  double worst = 0.0;
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) {
      Cx acc{0, 0};
      for (int c = 0; c < dim; ++c) acc = add(acc, mul(m[i * dim + c], conj(m[j * dim + c])));
      const Cx d = sub(acc, Cx{i == j ? 1.0 : 0.0, 0});
      const double dev = std::hypot(d.re, d.im);
      if (std::isnan(dev)) return NAN;
      if (dev > worst) worst = dev;
    }
  return worst;
}

bool is_zero(Cx a) { return a.re == 0.0 && a.im == 0.0; }
bool is_one(Cx a) { return a.re == 1.0 && a.im == 0.0; }

void push_coef(Lowered* L, const Cx* c, int count) {
  for (int i = 0; i < count; ++i) {
    L->coef.push_back(c[i].re);
    L->coef.push_back(c[i].im);
  }
}

// Lower a validated dense matrix with MSB-first targets to the cheapest op.
void lower_matrix(const Cx* m, int dim, const uint32_t* tq, uint64_t ctrl, Lowered* L) {
  Op& op = L->op;
  std::memset(&op, 0, sizeof(op));
  op.ctrl = ctrl;
  const int k = dim == 2 ? 1 : dim == 4 ? 2 : dim == 8 ? 3 : dim == 16 ? 4 : 5;
  uint64_t tmask = 0;
  for (int i = 0; i < k; ++i) tmask |= 1ull << tq[i];
  bool diag = true;
  for (int i = 0; i < dim && diag; ++i)
    for (int j = 0; j < dim; ++j)
      if (i != j && !is_zero(m[i * dim + j])) {
        diag = false;
        break;
      }
  if (diag) {
    // diag(1, ..., 1, c): phase on the all-ones corner
    bool corner = true;
    for (int i = 0; i + 1 < dim; ++i)
      if (!is_one(m[i * dim + i])) corner = false;
    const Cx c = m[dim * dim - 1];
    L->nondiag = 0;
    L->diag = tmask | ctrl;
    if (corner) {
      op.mask = tmask | ctrl;
      op.ctrl = 0;
      if (c.re == -1.0 && c.im == 0.0) {
        op.type = OP_NEG;
      } else {
        op.type = OP_CPHASE;
        push_coef(L, &c, 1);
      }
      return;
    }
    if (k <= 3) {
      op.type = OP_DIAG;
      op.nq = (uint8_t)k;
      for (int i = 0; i < k; ++i) op.q[i] = (uint8_t)tq[i];
      Cx d[8];
      for (int i = 0; i < dim; ++i) d[i] = m[i * dim + i];
      push_coef(L, d, dim);
      return;
    }
  }
  // controlled blocks: a 2q matrix I (+) U with the MSB as control -> 1q with control
  if (dim == 4 && is_one(m[0]) && is_zero(m[1]) && is_zero(m[2]) && is_zero(m[3]) && is_zero(m[4]) &&
      is_one(m[5]) && is_zero(m[6]) && is_zero(m[7]) && is_zero(m[8]) && is_zero(m[9]) && is_zero(m[12]) &&
      is_zero(m[13])) {
    const Cx u[4] = {m[10], m[11], m[14], m[15]};
    uint32_t t1 = tq[1];
    lower_matrix(u, 2, &t1, ctrl | (1ull << tq[0]), L);
    return;
  }
  // Toffoli / controlled-controlled-U pattern (8x8 identity except the last 2x2 block)
  if (dim == 8) {
    bool cc = true;
    for (int i = 0; i < 8 && cc; ++i)
      for (int j = 0; j < 8; ++j) {
        if (i >= 6 && j >= 6) continue;
        const Cx v = m[i * 8 + j];
        if (i == j ? !is_one(v) : !is_zero(v)) {
          cc = false;
          break;
        }
      }
    if (cc) {
      const Cx u[4] = {m[54], m[55], m[62], m[63]};
      uint32_t t2 = tq[2];
      lower_matrix(u, 2, &t2, ctrl | (1ull << tq[0]) | (1ull << tq[1]), L);
      return;
    }
  }
  L->nondiag = tmask;
  L->diag = ctrl;
  if (dim == 2) {
    op.nq = 1;
    op.q[0] = (uint8_t)tq[0];
    if (is_zero(m[0]) && is_one(m[1]) && is_one(m[2]) && is_zero(m[3])) {
      op.type = OP_X;
      return;
    }
    op.type = OP_1Q;
    push_coef(L, m, 4);
    return;
  }
  if (dim == 4) {
    op.type = OP_2Q;
    op.nq = 2;
    op.q[0] = (uint8_t)tq[0];
    op.q[1] = (uint8_t)tq[1];
    push_coef(L, m, 16);
    return;
  }
  op.type = OP_KQ;
  op.nq = (uint8_t)k;
  for (int i = 0; i < k; ++i) op.q[i] = (uint8_t)tq[i];
  push_coef(L, m, dim * dim);
}

}  // namespace

int gate_matrix_dense(const aleph_b200_instr& g, const double* pool, uint64_t pool_len, double* out, int* dim,
                      aleph_b200_error_info* e) {
  Cx m[8][8];
  const int d = matrix_of(g, pool, pool_len, m, e);
  if (d == 0) return e->status ? e->status : ALEPH_B200_UNSUPPORTED_GATE;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      out[2 * (i * d + j)] = m[i][j].re;
      out[2 * (i * d + j) + 1] = m[i][j].im;
    }
  *dim = d;
  return ALEPH_B200_OK;
}

const char* gate_name(uint32_t kind) {
  static const char* names[] = {"H",   "X",   "Y",   "Z",   "S",     "Sdg",     "T",       "Tdg",
                                "Rx",  "Ry",  "Rz",  "Phase", "U3",  "Cnot",    "Cz",      "Swap",
                                "Iswap", "IswapDg", "CRx", "CRy", "CRz", "Toffoli", "Ccz", "Unitary1q",
                                "Unitary2q", "UnitaryKq", "Unitary1qDiag", "Unitary2qDiag"};
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

int lower_gate(const aleph_b200_instr& g, uint32_t n, const double* pool, uint64_t pool_len, Lowered* L,
               aleph_b200_error_info* e, bool tiled) {
  const int expected = arity(g);
  if (expected < 0) {
    set_kind(e, gate_name(g.kind));
    return fail(e, ALEPH_B200_UNSUPPORTED_GATE);
  }
  if ((uint32_t)expected != g.num_qubits) {
    set_kind(e, gate_name(g.kind));
    e->expected = (uint32_t)expected;
    e->got = g.num_qubits;
    return fail(e, ALEPH_B200_ARITY_MISMATCH);
  }
  if (g.num_qubits > 8 || g.num_controls > 8) {
    set_kind(e, "record");
    return fail(e, ALEPH_B200_INVALID_ARGUMENT);
  }
  uint32_t seen[16];
  uint32_t ns = 0;
  uint64_t ctrl = 0;
  for (uint32_t i = 0; i < g.num_qubits + g.num_controls; ++i) {
    const uint32_t q = i < g.num_qubits ? g.qubits[i] : g.controls[i - g.num_qubits];
    if (q >= n) {
      e->qubit = q;
      e->num_qubits = n;
      return fail(e, ALEPH_B200_QUBIT_OUT_OF_RANGE);
    }
    for (uint32_t j = 0; j < ns; ++j)
      if (seen[j] == q) {
        e->qubit = q;
        return fail(e, ALEPH_B200_DUPLICATE_QUBIT);
      }
    seen[ns++] = q;
    if (i >= g.num_qubits) ctrl |= 1ull << q;
  }
  if (tiled && g.kind == ALEPH_GATE_UNITARYKQ) {
    // a gate of a TiledBlock goes through Gate::matrix() only
    // (dispatch_tile_kernel, crates/aleph-sv/src/backend.rs:265-299), and a
    // UnitaryKq has no fixed-size matrix there: UnsupportedGate
    set_kind(e, gate_name(g.kind));
    return fail(e, ALEPH_B200_UNSUPPORTED_GATE);
  }
  if (g.kind == ALEPH_GATE_UNITARYKQ) {
    // validate_unitary_kq, crates/aleph-sv/src/validation.rs:113-155
    const uint32_t k = g.aux;
    if (k < 2 || k > 5) {
      set_kind(e, "UnitaryKq width");
      return fail(e, ALEPH_B200_INVALID_STATE);
    }
    if (g.num_controls) {
      set_kind(e, "controlled UnitaryKq");
      return fail(e, ALEPH_B200_UNSUPPORTED_GATE);
    }
    const uint64_t w = 1ull << k;
    if (g.data_len != w * w) {
      set_kind(e, "UnitaryKq length");
      return fail(e, ALEPH_B200_INVALID_STATE);
    }
    if (!pool || g.data_offset + g.data_len > pool_len) {
      set_kind(e, "matrix pool");
      return fail(e, ALEPH_B200_INVALID_ARGUMENT);
    }
    const Cx* d = reinterpret_cast<const Cx*>(pool + 2 * g.data_offset);
    for (uint64_t i = 0; i < w * w; ++i)
      if (!std::isfinite(d[i].re) || !std::isfinite(d[i].im)) {
        set_kind(e, "UnitaryKq");
        return fail(e, ALEPH_B200_NON_FINITE_PARAM);
      }
    double dev2 = 0.0;
    for (uint64_t i = 0; i < w; ++i)
      for (uint64_t j = 0; j <= i; ++j) {
        Cx s{0, 0};
        for (uint64_t c = 0; c < w; ++c) s = add(s, mul(d[i * w + c], conj(d[j * w + c])));
        const Cx df = sub(s, Cx{i == j ? 1.0 : 0.0, 0});
        const double er = df.re * df.re + df.im * df.im;
        if (!std::isfinite(er)) {
          e->value = er;
          return fail(e, ALEPH_B200_NON_UNITARY_MATRIX);
        }
        dev2 = std::max(dev2, er);
      }
    if (dev2 > kTol * kTol) {
      e->value = std::sqrt(dev2);
      return fail(e, ALEPH_B200_NON_UNITARY_MATRIX);
    }
    L->record = 0;
    lower_matrix(d, (int)w, g.qubits, 0, L);
    return ALEPH_B200_OK;
  }
  Cx m[8][8];
  const int dim = matrix_of(g, pool, pool_len, m, e);
  if (dim == 0) return e->status;
  Cx flat[64];
  for (int i = 0; i < dim; ++i)
    for (int j = 0; j < dim; ++j) flat[i * dim + j] = m[i][j];
  if (tiled) {
    // TiledBlock gates: the tile kernels take 2x2 and 4x4 matrices; an 8x8
    // is UnsupportedGate, and no unitarity check is made (backend.rs:265-299)
    if (dim > 4) {
      set_kind(e, gate_name(g.kind));
      return fail(e, ALEPH_B200_UNSUPPORTED_GATE);
    }
    lower_matrix(flat, dim, g.qubits, ctrl, L);
    return ALEPH_B200_OK;
  }
  const double dev = unitarity_deviation(flat, dim);
  if (!std::isfinite(dev) || dev > kTol) {
    e->value = dev;
    return fail(e, ALEPH_B200_NON_UNITARY_MATRIX);
  }
  lower_matrix(flat, dim, g.qubits, ctrl, L);
  return ALEPH_B200_OK;
}

int lower_diagonal_phase(const aleph_b200_phase_term* terms, uint64_t n_terms, const uint64_t* conds, uint64_t n_conds,
                         Lowered* L, aleph_b200_error_info* e) {
  std::memset(&L->op, 0, sizeof(L->op));
  L->op.type = OP_POLY;
  L->op.aux = (uint32_t)n_terms;
  uint64_t support = 0;
  for (uint64_t t = 0; t < n_terms; ++t) {
    if ((uint64_t)terms[t].cond_offset + terms[t].cond_count > n_conds || (!conds && terms[t].cond_count)) {
      set_kind(e, "diagonal phase conds");
      return fail(e, ALEPH_B200_INVALID_ARGUMENT);
    }
    L->poly_angle.push_back(terms[t].angle);
    L->poly_cnt.push_back(terms[t].cond_count);
    for (uint32_t c = 0; c < terms[t].cond_count; ++c) {
      L->poly_conds.push_back(conds[terms[t].cond_offset + c]);
      support |= conds[terms[t].cond_offset + c];
    }
  }
  L->nondiag = 0;
  L->diag = support;
  return ALEPH_B200_OK;
}

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------
namespace {

uint32_t append_op(Plan* P, const Lowered& L, Op op) {
  op.coef = (uint32_t)(P->coef.size() / 2);
  P->coef.insert(P->coef.end(), L.coef.begin(), L.coef.end());
  if (op.type == OP_POLY) {
    op.mask = P->poly_angle.size();
    uint32_t off = 0;
    for (size_t t = 0; t < L.poly_angle.size(); ++t) {
      P->poly_angle.push_back(L.poly_angle[t]);
      P->poly_off.push_back((uint32_t)P->poly_conds.size());
      P->poly_cnt.push_back(L.poly_cnt[t]);
      for (uint32_t c = 0; c < L.poly_cnt[t]; ++c) P->poly_conds.push_back(L.poly_conds[off + c]);
      off += L.poly_cnt[t];
    }
  }
  P->ops.push_back(op);
  return (uint32_t)(P->ops.size() - 1);
}

// Cost-model features of a pass from the ops it applies.
void count_ops(const std::vector<const Lowered*>& ops, Pass* ps) {
  for (const Lowered* L : ops) {
    switch (L->op.type) {  // a complex multiply-add is 4 real ones
      case OP_1Q: ps->fma_per_amp += 8; break;
      case OP_2Q: ps->fma_per_amp += 16; break;
      case OP_KQ: ps->fma_per_amp += 4u << L->op.nq; break;
      case OP_CPHASE: case OP_DIAG: case OP_POLY: ps->fma_per_amp += 4; break;
      default: break;  // X and sign flips move or negate
    }
    if (L->nondiag) {
      ++ps->dense_ops;
      if (L->nondiag & 0x1Full) ++ps->lane_ops;
    } else {
      ++ps->diag_ops;
    }
  }
}

// Swap the operand order of a 4x4 matrix (MSB <-> LSB).
void swap_2q_operands(std::vector<double>& c) {
  std::vector<double> out(c.size());
  auto sw = [](int k) { return ((k & 1) << 1) | (k >> 1); };
  for (int r = 0; r < 4; ++r)
    for (int cc = 0; cc < 4; ++cc) {
      const int src = 2 * (4 * r + cc), dst = 2 * (4 * sw(r) + sw(cc));
      out[dst] = c[src];
      out[dst + 1] = c[src + 1];
    }
  c = out;
}

// ---- pair fusion (warp-tile passes) ------------------------------------------
// A tile pass applies its gates one at a time in registers, so its arithmetic
// is the sum of the gates': 8 FP64 multiply-adds per amplitude for a dense
// one-qubit gate, 16 for a dense two-qubit one, one or two for a diagonal.
// In FP64 the pass is bound by that arithmetic. A two-qubit gate together
// with the one-qubit gates around it on its two qubits is one 4x4 (16 per
// amplitude): in a brickwall, the one-qubit layers on both sides of a CZ,
// four dense gates (32) for one 4x4 (16).
//
// The rule, in gate order: one-qubit gates wait on their qubit. A gate on
// exactly two qubits a, b opens a block that takes the waiting one-qubit
// gates of a and b, itself, then every later gate on a and/or b alone, until
// a gate touches a or b together with another qubit. The block is then
// emitted as one 4x4 when its gates cost at least 24 per amplitude; otherwise
// its gates are emitted unchanged and the one-qubit gates at its end wait
// again on their qubits (so a CZ between two already-absorbed layers leaves
// the next layer to the next block). This is the idea of Fuse2q
// (crates/aleph-ir/src/passes/fuse_2q.rs) with a cost rule for register tiles.
void apply_local(const Lowered& L, const uint32_t* bq, Cx* s);

namespace {

int tile_cost(const Lowered& L) {
  switch (L.op.type) {
    case OP_1Q: return 8;
    case OP_2Q: return 16;
    case OP_X: case OP_NEG: return 1;
    case OP_CPHASE: case OP_DIAG: return 2;
    default: return 32;
  }
}

constexpr int kFuseMinCost = 24;

// The 4x4 of an op on qubits {a (matrix MSB), b (LSB)}, right-multiplied into m:
// m := op * m.
void fold_into_4x4(const Lowered& L, uint32_t a, uint32_t b, Cx* m) {
  const uint32_t bq[6] = {b, a, 60, 61, 62, 63};  // local bit 0 = b, bit 1 = a
  Cx out[16];
  for (uint32_t c = 0; c < 4; ++c) {
    Cx s[64];
    for (auto& x : s) x = Cx{0, 0};
    for (uint32_t r = 0; r < 4; ++r) s[r] = m[r * 4 + c];
    apply_local(L, bq, s);
    for (uint32_t r = 0; r < 4; ++r) out[r * 4 + c] = s[r];
  }
  for (int i = 0; i < 16; ++i) m[i] = out[i];
}

bool fusable_type(const Lowered& L) {
  return !L.is_measure && !L.is_permute && L.op.type != OP_POLY && L.op.type != OP_KQ;
}

}  // namespace

std::vector<const Lowered*> fuse_pairs(const std::vector<const Lowered*>& seg, std::deque<Lowered>& store) {
  struct Block {
    uint32_t a, b;
    Cx m[16];
    std::vector<const Lowered*> members;
    int cost = 0;
    uint32_t record = 0;
  };
  std::vector<const Lowered*> out;
  out.reserve(seg.size());
  std::vector<std::vector<size_t>> waiting(kMaxQubits);  // out indices of one-qubit gates waiting per qubit
  std::vector<int> open(kMaxQubits, -1);
  std::vector<Block> blocks;
  auto close = [&](uint32_t q) {
    const int k = open[q];
    if (k < 0) return;
    Block& B = blocks[(size_t)k];
    open[B.a] = open[B.b] = -1;
    if (B.cost >= kFuseMinCost) {
      store.emplace_back();
      Lowered& F = store.back();
      std::memset(&F.op, 0, sizeof(Op));
      F.op.type = OP_2Q;
      F.op.nq = 2;
      F.op.q[0] = (uint8_t)B.a;
      F.op.q[1] = (uint8_t)B.b;
      push_coef(&F, B.m, 16);
      F.nondiag = (1ull << B.a) | (1ull << B.b);
      F.diag = 0;
      F.record = B.record;
      F.gates = 0;
      for (const Lowered* L : B.members) F.gates += L->gates ? L->gates : 1;
      out.push_back(&F);
      waiting[B.a].clear();
      waiting[B.b].clear();
      return;
    }
    // not worth a 4x4: the gates go out as they came; the one-qubit gates
    // after the block's last two-qubit gate wait again on their qubits
    size_t last2 = 0;
    for (size_t i = 0; i < B.members.size(); ++i)
      if (__builtin_popcountll(B.members[i]->nondiag | B.members[i]->diag) == 2) last2 = i;
    waiting[B.a].clear();
    waiting[B.b].clear();
    for (size_t i = 0; i < B.members.size(); ++i) {
      out.push_back(B.members[i]);
      if (i > last2) {
        const uint64_t t = B.members[i]->nondiag | B.members[i]->diag;
        waiting[(uint32_t)__builtin_ctzll(t)].push_back(out.size() - 1);
      }
    }
  };
  for (const Lowered* L : seg) {
    const uint64_t touched = L->nondiag | L->diag;
    const int width = __builtin_popcountll(touched);
    if (fusable_type(*L) && width == 1) {
      const uint32_t q = (uint32_t)__builtin_ctzll(touched);
      const int k = open[q];
      if (k >= 0) {
        Block& B = blocks[(size_t)k];
        fold_into_4x4(*L, B.a, B.b, B.m);
        B.members.push_back(L);
        B.cost += tile_cost(*L);
      } else {
        out.push_back(L);
        waiting[q].push_back(out.size() - 1);
      }
      continue;
    }
    if (fusable_type(*L) && width == 2) {
      const uint32_t lo = (uint32_t)__builtin_ctzll(touched), hi = 63u - (uint32_t)__builtin_clzll(touched);
      if (open[lo] >= 0 && open[lo] == open[hi]) {  // another gate on the same pair
        Block& B = blocks[(size_t)open[lo]];
        fold_into_4x4(*L, B.a, B.b, B.m);
        B.members.push_back(L);
        B.cost += tile_cost(*L);
        continue;
      }
      close(lo);
      close(hi);
      Block B;
      B.a = hi;
      B.b = lo;
      for (int i = 0; i < 16; ++i) B.m[i] = Cx{(i % 5) == 0 ? 1.0 : 0.0, 0.0};
      B.record = L->record;
      for (uint32_t q : {hi, lo}) {
        for (size_t idx : waiting[q]) {
          const Lowered* W = out[idx];
          fold_into_4x4(*W, B.a, B.b, B.m);
          B.members.push_back(W);
          B.cost += tile_cost(*W);
          out[idx] = nullptr;
        }
        waiting[q].clear();
      }
      fold_into_4x4(*L, B.a, B.b, B.m);
      B.members.push_back(L);
      B.cost += tile_cost(*L);
      blocks.push_back(std::move(B));
      open[hi] = open[lo] = (int)blocks.size() - 1;
      continue;
    }
    for (uint32_t q = 0; q < kMaxQubits; ++q)
      if ((touched >> q) & 1) {
        close(q);
        waiting[q].clear();
      }
    out.push_back(L);
  }
  for (uint32_t q = 0; q < kMaxQubits; ++q) close(q);
  std::vector<const Lowered*> compact;
  compact.reserve(out.size());
  for (const Lowered* L : out)
    if (L) compact.push_back(L);
  return compact;
}

int plan_segment_tiles(const std::vector<const Lowered*>& seg, uint32_t n, uint32_t R, Plan* P) {
  std::vector<const Lowered*> pending = seg;
  while (!pending.empty()) {
    const Lowered* head = pending.front();
    if (head->op.type == OP_KQ) {
      Pass ps{};
      ps.kind = PASS_KQ;
      ps.tile.n = n;
      ps.tile.op_begin = append_op(P, *head, head->op);
      ps.tile.op_count = 1;
      ps.record = head->record;
      ps.gates = 1;
      ps.dense_ops = 1;
      P->passes.push_back(ps);
      pending.erase(pending.begin());
      continue;
    }
    uint64_t hi = 0;          // register qubits chosen so far
    uint32_t nhi = 0;
    uint64_t blocked_full = 0, blocked_diag = 0;
    std::vector<const Lowered*> take, rest;
    for (const Lowered* L : pending) {
      bool ok = !(L->nondiag & (blocked_full | blocked_diag)) && !(L->diag & blocked_full);
      uint64_t need = 0;
      if (ok && L->op.type == OP_KQ) ok = false;
      if (ok && L->nondiag) {
        need = (L->nondiag >> 5 << 5) & ~hi;
        if (nhi + (uint32_t)__builtin_popcountll(need) > R) ok = false;
      }
      if (ok) {
        hi |= need;
        nhi += (uint32_t)__builtin_popcountll(need);
        take.push_back(L);
      } else {
        blocked_full |= L->nondiag;
        blocked_diag |= L->diag;
        rest.push_back(L);
      }
    }
    // register qubits: the chosen ones, padded with the lowest unused qubits >= 5
    TilePass tp{};
    tp.n = n;
    tp.R = R;
    uint32_t j = 0;
    for (uint32_t q = 5; q < n && j < R; ++q)
      if ((hi >> q) & 1) tp.hq[j++] = q;
    for (uint32_t q = 5; q < n && j < R; ++q)
      if (!((hi >> q) & 1)) {
        tp.hq[j++] = q;
        hi |= 1ull << q;
      }
    auto slot = [&](uint32_t q) -> uint8_t {
      if (q < 5) return (uint8_t)q;
      for (uint32_t i = 0; i < R; ++i)
        if (tp.hq[i] == q) return (uint8_t)(5 + i);
      return 255;
    };
    tp.op_begin = (uint32_t)P->ops.size();
    // Split a global qubit mask into the bits outside the register qubits and
    // an R-bit mask over the register slots (tested per element in the kernel).
    auto split = [&](uint64_t m, uint64_t* rest, uint8_t* creg) {
      *rest = m;
      *creg = 0;
      for (uint32_t j = 0; j < R; ++j)
        if ((m >> tp.hq[j]) & 1) {
          *creg |= (uint8_t)(1u << j);
          *rest &= ~(1ull << tp.hq[j]);
        }
    };
    for (const Lowered* L : take) {
      Op op = L->op;
      if (op.type == OP_NEG || op.type == OP_CPHASE) {
        split(op.mask, &op.mask, &op.creg);
        op.ctrl = 0;
      } else if (op.type != OP_POLY) {
        split(op.ctrl, &op.ctrl, &op.creg);
      }
      if (op.type == OP_DIAG) {
        op.dsrc = 0;
        for (int i = 0; i < op.nq; ++i) {
          const uint8_t s = slot(op.q[i]);
          if (s >= 5 && s != 255) {
            op.dsrc |= (uint8_t)(1u << i);
            op.q[3 + i] = (uint8_t)(s - 5);
          }
        }
      }
      if (op.type == OP_1Q || op.type == OP_X) {
        op.a = slot(op.q[0]);
        append_op(P, *L, op);
      } else if (op.type == OP_2Q) {
        uint8_t sa = slot(op.q[0]), sb = slot(op.q[1]);
        if (sa < sb) {
          Lowered tmp = *L;
          swap_2q_operands(tmp.coef);
          std::swap(op.q[0], op.q[1]);
          op.a = sb;
          op.b = sa;
          append_op(P, tmp, op);
        } else {
          op.a = sa;
          op.b = sb;
          append_op(P, *L, op);
        }
      } else {
        append_op(P, *L, op);
      }
    }
    tp.op_count = (uint32_t)P->ops.size() - tp.op_begin;
    if (take.empty()) return ALEPH_B200_OPTIMIZATION;  // no progress: the head op fits no tile
    Pass ps{};
    ps.kind = PASS_TILE;
    ps.tile = tp;
    ps.record = take.empty() ? 0 : take.front()->record;
    ps.gates = 0;
    for (const Lowered* L : take) ps.gates += L->gates ? L->gates : 1;
    count_ops(take, &ps);
    P->passes.push_back(ps);
    pending.swap(rest);
  }
  return ALEPH_B200_OK;
}

// ---- tensor-core dense blocks ------------------------------------------------
// Apply a lowered op to a vector over the block qubits bq[0..6) (index bit b
// <-> qubit bq[b]); the op's qubits must all be block qubits, except for the
// diagonal-polynomial case where only the support matters.
void apply_local(const Lowered& L, const uint32_t* bq, Cx* s) {
  auto lbit = [&](uint32_t q) -> uint32_t {
    for (uint32_t b = 0; b < 6; ++b)
      if (bq[b] == q) return b;
    return 63;
  };
  auto lmask = [&](uint64_t m) -> uint32_t {
    uint32_t r = 0;
    for (uint32_t q = 0; q < 64; ++q)
      if ((m >> q) & 1) r |= 1u << lbit(q);
    return r;
  };
  auto gidx = [&](uint32_t x) -> uint64_t {
    uint64_t g = 0;
    for (uint32_t b = 0; b < 6; ++b)
      if ((x >> b) & 1) g |= 1ull << bq[b];
    return g;
  };
  const Op& op = L.op;
  const Cx* c = reinterpret_cast<const Cx*>(L.coef.data());
  switch (op.type) {
    case OP_NEG:
    case OP_CPHASE: {
      const uint32_t m = lmask(op.mask);
      const Cx f = op.type == OP_NEG ? Cx{-1, 0} : c[0];
      for (uint32_t x = 0; x < 64; ++x)
        if ((x & m) == m) s[x] = mul(f, s[x]);
      return;
    }
    case OP_DIAG: {
      const uint32_t cm = lmask(op.ctrl);
      for (uint32_t x = 0; x < 64; ++x) {
        if ((x & cm) != cm) continue;
        uint32_t idx = 0;
        for (int i = 0; i < op.nq; ++i) idx = (idx << 1) | ((x >> lbit(op.q[i])) & 1);
        s[x] = mul(c[idx], s[x]);
      }
      return;
    }
    case OP_POLY: {
      for (uint32_t x = 0; x < 64; ++x) {
        const uint64_t g = gidx(x);
        double phi = 0.0;
        size_t off = 0;
        for (size_t t = 0; t < L.poly_angle.size(); ++t) {
          bool all = true;
          for (uint32_t k = 0; k < L.poly_cnt[t]; ++k)
            if ((__builtin_popcountll(L.poly_conds[off + k] & g) & 1) == 0) all = false;
          off += L.poly_cnt[t];
          if (all) phi += L.poly_angle[t];
        }
        s[x] = mul(Cx{std::cos(phi), std::sin(phi)}, s[x]);
      }
      return;
    }
    default: break;
  }
  // dense: k targets MSB-first, controls
  const int k = op.type == OP_2Q ? 2 : op.type == OP_KQ ? op.nq : 1;
  const uint32_t dim = 1u << k;
  const uint32_t cm = lmask(op.ctrl);
  uint32_t tmask = 0, off[32];
  for (int i = 0; i < k; ++i) tmask |= 1u << lbit(op.q[i]);
  for (uint32_t r = 0; r < dim; ++r) {
    uint32_t o = 0;
    for (int p = 0; p < k; ++p)
      if ((r >> p) & 1) o |= 1u << lbit(op.q[k - 1 - p]);
    off[r] = o;
  }
  for (uint32_t base = 0; base < 64; ++base) {
    if ((base & tmask) || (base & cm) != cm) continue;
    Cx v[32], w[32];
    for (uint32_t r = 0; r < dim; ++r) v[r] = s[base | off[r]];
    for (uint32_t r = 0; r < dim; ++r) {
      if (op.type == OP_X) {
        w[r] = v[r ^ 1];
        continue;
      }
      Cx acc{0, 0};
      for (uint32_t cc = 0; cc < dim; ++cc) acc = add(acc, mul(c[r * dim + cc], v[cc]));
      w[r] = acc;
    }
    for (uint32_t r = 0; r < dim; ++r) s[base | off[r]] = w[r];
  }
}

// One block pass drawn from the pending ops: the ops fused into the block
// (`take`), the diagonal ops applied after it in the epilogue (`post`) and the
// ops left for later passes (`rest`, in order). With `fixed`, the block
// qubits are `fixedB`; otherwise they grow first-come up to 6 qubits. An op
// joins only if it commutes past every op deferred before it.
struct BlockTake {
  uint64_t B = 0;
  std::vector<const Lowered*> take, post, rest;
  // Ops consumed, each weighted by its age: 1 / (1 + (record - base) / 64),
  // base = the oldest pending record. Preferring old ops keeps the frontier
  // level; on the n=32 depth-40 brickwall it plans 67 passes where a plain
  // count plans 70 (a planner model swept the scale: 64-128 best).
  double score(uint32_t base) const {
    if (take.empty()) return 0.0;
    double s = 0.0;
    for (const Lowered* L : take) s += 1.0 / (1.0 + (double)(L->record - base) / 64.0);
    for (const Lowered* L : post) s += 1.0 / (1.0 + (double)(L->record - base) / 64.0);
    return s;
  }
};

void block_take(const std::vector<const Lowered*>& pending, uint64_t fixedB, bool fixed, BlockTake* out) {
  uint64_t B = fixed ? fixedB : 0, bf = 0, bd = 0, post_lock = 0;
  auto fits = [&](uint64_t supp) {
    return fixed ? (supp & ~fixedB) == 0 : __builtin_popcountll(B | supp) <= 6;
  };
  for (const Lowered* L : pending) {
    const uint64_t supp = L->nondiag | L->diag;
    if (L->nondiag) {
      if (!(L->nondiag & (bf | bd | post_lock)) && !(L->diag & bf) && fits(supp)) {
        B |= supp;
        out->take.push_back(L);
        continue;
      }
    } else if (!(L->diag & bf)) {
      if (fits(supp)) {
        B |= supp;
        out->take.push_back(L);
        continue;
      }
      if (B != 0 && out->post.size() < 48) {  // the block kernel caches up to 48 post ops
        out->post.push_back(L);
        post_lock |= supp;
        continue;
      }
    }
    bf |= L->nondiag;
    bd |= L->diag;
    out->rest.push_back(L);
  }
  out->B = B;
}

// One block pass's fused unitary, still to be built: its ops, its qubits and
// the byte offset of its image in the plan.
struct BlockJob {
  std::vector<const Lowered*> take;
  uint32_t bq[6];
  uint32_t mat;
};

// Fuse each job's ops into a 64x64 unitary (columns = images of the basis
// vectors, in FP64), lay it out as W = [[Re U, -Im U], [Im U, Re U]] and write
// the split-BF16 image. The jobs are independent: they run on host threads.
void build_block_images(const std::vector<BlockJob>& jobs, Plan* P) {
  if (jobs.empty()) return;
  P->block_images.resize(P->block_images.size() + jobs.size() * kBlockImageBytes);
  auto build = [&](size_t k) {
    const BlockJob& J = jobs[k];
    std::vector<Cx> U(64 * 64);
    for (uint32_t col = 0; col < 64; ++col) {
      Cx s[64];
      for (uint32_t x = 0; x < 64; ++x) s[x] = Cx{x == col ? 1.0 : 0.0, 0.0};
      for (const Lowered* L : J.take) apply_local(*L, J.bq, s);
      for (uint32_t x = 0; x < 64; ++x) U[x * 64 + col] = s[x];
    }
    std::vector<double> W(128 * 128);
    for (uint32_t r = 0; r < 64; ++r)
      for (uint32_t c = 0; c < 64; ++c) {
        const Cx u = U[r * 64 + c];
        W[r * 128 + c] = u.re;
        W[r * 128 + 64 + c] = -u.im;
        W[(64 + r) * 128 + c] = u.im;
        W[(64 + r) * 128 + 64 + c] = u.re;
      }
    build_block_image(W.data(), P->block_images.data() + J.mat);
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = std::min<size_t>(jobs.size(), hw ? std::min(hw, 16u) : 1u);
  if (nt <= 1) {
    for (size_t k = 0; k < jobs.size(); ++k) build(k);
    return;
  }
  std::vector<std::thread> ws;
  for (size_t t = 0; t < nt; ++t)
    ws.emplace_back([&, t] {
      for (size_t k = t; k < jobs.size(); k += nt) build(k);
    });
  for (auto& w : ws) w.join();
}

int plan_segment_blocks(const std::vector<const Lowered*>& seg, uint32_t n, uint32_t R, bool window_search,
                        Plan* P) {
  std::vector<const Lowered*> pending = seg;
  std::vector<BlockJob> jobs;
  while (!pending.empty()) {
    // Candidates: the first-come block, and (window_search) every window of 6
    // consecutive qubits; the one with the highest age-weighted op count wins
    // (ties keep the earlier candidate). On a brickwall the windows follow
    // the light cone, which first-come growth does not.
    const uint32_t base = pending.front()->record;
    BlockTake best;
    block_take(pending, 0, false, &best);
    double best_score = best.score(base);
    if (window_search)
      for (uint32_t a = 0; a + 6 <= n; ++a) {
        BlockTake c;
        block_take(pending, 0x3Full << a, true, &c);
        const double s = c.score(base);
        if (s > best_score) {
          best = std::move(c);
          best_score = s;
        }
      }
    uint64_t B = best.B;
    std::vector<const Lowered*>& take = best.take;
    std::vector<const Lowered*>& post = best.post;
    std::vector<const Lowered*>& rest = best.rest;
    if (take.empty()) {
      // the head op does not fit a 6-qubit block: run it on the CUDA cores
      std::vector<const Lowered*> one{pending.front()};
      if (int s = plan_segment_tiles(one, n, R, P)) return s;
      pending.erase(pending.begin());
      continue;
    }
    // pad the block to 6 qubits with the lowest unused qubits
    for (uint32_t q = 0; q < n && __builtin_popcountll(B) < 6; ++q) B |= 1ull << q;
    uint32_t bq[6], nb = 0;
    for (uint32_t q = 0; q < n; ++q)
      if ((B >> q) & 1) bq[nb++] = q;
    Pass ps{};
    ps.kind = PASS_BLOCK;
    ps.block.n = n;
    for (int j = 0; j < 6; ++j) ps.block.bq[j] = bq[j];
    ps.block.mat = (uint32_t)(P->block_images.size() + jobs.size() * kBlockImageBytes);
    jobs.push_back(BlockJob{take, {bq[0], bq[1], bq[2], bq[3], bq[4], bq[5]}, ps.block.mat});
    ps.block.post_begin = (uint32_t)P->ops.size();
    for (const Lowered* L : post) append_op(P, *L, L->op);
    ps.block.post_count = (uint32_t)P->ops.size() - ps.block.post_begin;
    ps.block.fold = 0;
    for (const Lowered* L : post) {
      const Op& op = L->op;
      if ((op.type == OP_CPHASE && __builtin_popcountll(op.mask & B) <= 1) ||
          (op.type == OP_DIAG && op.nq == 1 && !((B >> op.q[0]) & 1) && !(op.ctrl & B)))
        ps.block.fold = 1;
    }
    ps.record = take.front()->record;
    ps.gates = (uint32_t)(take.size() + post.size());
    count_ops(take, &ps);
    ps.lane_ops = 0;  // a block has no lane shuffles
    ps.diag_ops += (uint32_t)post.size();
    P->passes.push_back(ps);
    pending.swap(rest);
  }
  build_block_images(jobs, P);
  return ALEPH_B200_OK;
}

}  // namespace

// A cycle c_0 -> c_1 -> ... -> c_{m-1} -> c_0 of pi is alpha o beta with the
// reflections beta(c_i) = c_{-i} and alpha(c_i) = c_{1-i} (indices mod m), both
// involutions; alpha is applied first (P_beta P_alpha psi = psi o alpha o beta).
std::vector<std::vector<uint8_t>> split_into_involutions(const std::vector<uint32_t>& pi) {
  const uint32_t n = (uint32_t)pi.size();
  std::vector<uint8_t> alpha(n), beta(n);
  std::vector<bool> seen(n, false);
  bool alpha_id = true, beta_id = true;
  for (uint32_t s = 0; s < n; ++s) {
    if (seen[s]) continue;
    std::vector<uint32_t> cyc;
    for (uint32_t q = s; !seen[q]; q = pi[q]) {
      seen[q] = true;
      cyc.push_back(q);
    }
    const uint32_t m = (uint32_t)cyc.size();
    for (uint32_t i = 0; i < m; ++i) {
      beta[cyc[i]] = (uint8_t)cyc[(m - i) % m];
      alpha[cyc[i]] = (uint8_t)cyc[(m + 1 - i) % m];
      beta_id &= beta[cyc[i]] == cyc[i];
      alpha_id &= alpha[cyc[i]] == cyc[i];
    }
  }
  std::vector<std::vector<uint8_t>> out;
  if (!alpha_id) out.push_back(alpha);
  if (!beta_id) out.push_back(beta);
  return out;
}

int build_plan(const std::vector<Lowered>& ops, uint32_t n, const PlanOptions& o, Plan* P) {
  P->renormalize = o.renormalize;
  std::vector<const Lowered*> seg;
  int status = ALEPH_B200_OK;
  auto flush = [&]() {
    if (seg.empty() || status) return;
    if (n <= o.smem_max_n || n < 6) {
      Pass ps{};
      ps.kind = PASS_SMEM;
      ps.tile.n = n;
      ps.tile.op_begin = (uint32_t)P->ops.size();
      for (const Lowered* L : seg) append_op(P, *L, L->op);
      ps.tile.op_count = (uint32_t)P->ops.size() - ps.tile.op_begin;
      ps.record = seg.front()->record;
      ps.gates = (uint32_t)seg.size();
      count_ops(seg, &ps);
      P->passes.push_back(ps);
    } else {
      // a 2-qubit gate may need two register qubits: R >= 2 unless only one high qubit exists
      const uint32_t R = std::min<uint32_t>(std::max<uint32_t>(o.tile_r, 2), std::min<uint32_t>(5, n - 5));
      if (o.tensor_blocks && n >= 13) status = plan_segment_blocks(seg, n, R, o.block_window_search, P);
      else if (o.pair_fusion) {
        std::deque<Lowered> fused;
        status = plan_segment_tiles(fuse_pairs(seg, fused), n, R, P);
      } else {
        status = plan_segment_tiles(seg, n, R, P);
      }
    }
    seg.clear();
  };
  for (const Lowered& L : ops) {
    if (L.is_measure) {
      flush();
      Pass ps{};
      ps.kind = PASS_MEASURE;
      ps.qubit = L.measure_qubit;
      ps.record = L.record;
      P->passes.push_back(ps);
      ++P->n_measures;
    } else if (L.is_permute) {
      flush();
      Pass ps{};
      ps.kind = PASS_PERMUTE;
      for (uint32_t q = 0; q < n && q < kMaxQubits; ++q) ps.sigma[q] = L.sigma[q];
      ps.record = L.record;
      ps.gates = L.gates;
      P->passes.push_back(ps);
    } else {
      seg.push_back(&L);
    }
  }
  flush();
  for (Pass& ps : P->passes)
    if (ps.kind == PASS_TILE) ps.tile.occupancy = o.tile_occupancy;
  return status;
}

}  // namespace ab
