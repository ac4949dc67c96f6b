// sv_pipeline.cpp — TEST INFRASTRUCTURE and CPU BASELINE, not product code.
//
// CPU restatement of what `aleph run --backend sv` executes by default: the
// final-state CPU pass pipeline (PassPipeline::final_state_cpu_pipeline,
// crates/aleph-ir/src/passes/mod.rs:192-201) —
//   RelabelQubits -> CancelInversePairs -> Fuse1qRuns -> Fuse2q ->
//   FuseKq (max 4 qubits) -> TileBlock (tile_bits 15)
// — then the optimised circuit on the CPU `sv` backend, and a final
// unpermute when the relabelling fired (run_optimized_with_pipeline,
// crates/aleph-backend/src/lib.rs:353-389; CLI exec.rs:582).
//
// It exists to time the reference's default CPU path on the host cores
// (bench.py's CPU baseline and reference arm) and is held to the raw
// gate-by-gate oracle (sv_oracle.cpp) at 1e-12 by the CPU tests, which is the
// reference's own guarantee for the optimised path
// (crates/aleph-backend/tests/run_optimized_oracle.rs:18). Each pass cites the
// reference function it follows.
//
// Unlike sv_oracle.cpp this file is built with FMA contraction and
// vectorisation allowed (it is a timing path, compared at 1e-12, not
// bit-for-bit), and its loops run on OpenMP threads (ORACLE_THREADS, default
// all hardware threads), like the reference's rayon blocks. The reference's
// own kernels are AVX-512 Rust; these are portable C++, so this is a
// restatement of the reference CPU path, not the reference binary.
#include <immintrin.h>
#include <omp.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <thread>
#include <vector>

#include "../include/aleph_b200.h"

// from sv_oracle.cpp (same library)
extern "C" {
int orc_gate_matrix(const aleph_b200_instr* g, const double* pool, uint64_t pool_len, double* out, int* dim_out);
int orc_apply_diagonal_phase(double* amps, uint32_t n, const aleph_b200_phase_term* terms, uint64_t nt,
                             const uint64_t* conds, uint64_t n_conds);
int orc_unpermute(double* amps, uint32_t n, const uint32_t* perm);
int orc_measure(double* amps, uint32_t n, uint32_t qubit, double u, int* outcome_out, int* consumed);
}

namespace {

using C = std::complex<double>;

// Read on every parallel region, so a caller can time one run on one core
// and the next on all of them.
int threads() {
  const char* e = std::getenv("ORACLE_THREADS");
  int v = e ? std::atoi(e) : 0;
  if (v <= 0) v = (int)std::thread::hardware_concurrency();
  return v <= 0 ? 1 : v;
}

// ---- instructions ----------------------------------------------------------
struct PGate {
  uint32_t kind = 0;
  std::vector<uint32_t> q;  // operand order (q[0] = matrix MSB)
  std::vector<uint32_t> c;  // external controls
  double p[3] = {0, 0, 0};
  uint32_t k = 0;           // UnitaryKq width
  std::vector<C> data;      // Unitary*: the matrix / diagonal, row-major
};

enum class IK { Gate, Measure, Reset, Barrier, Diag, Tiled };

struct PInst {
  IK t = IK::Gate;
  PGate g;
  uint32_t qubit = 0, clbit = 0;         // Measure / Reset
  std::vector<uint32_t> qs;              // Barrier
  std::vector<aleph_b200_phase_term> terms;  // DiagonalPhase (cond offsets into conds)
  std::vector<uint64_t> conds;
  uint32_t dp_n = 0;
  std::vector<PGate> gates;              // TiledBlock
  uint32_t tile_bits = 0;
};

bool is_unitary_kind(uint32_t k) { return k >= ALEPH_GATE_UNITARY1Q && k <= ALEPH_GATE_UNITARY2QDIAG; }

// Gate::arity (crates/aleph-core/src/gate/kinds.rs:110-152)
uint32_t arity(const PGate& g) {
  switch (g.kind) {
    case ALEPH_GATE_CNOT: case ALEPH_GATE_CZ: case ALEPH_GATE_SWAP: case ALEPH_GATE_ISWAP:
    case ALEPH_GATE_ISWAPDG: case ALEPH_GATE_CRX: case ALEPH_GATE_CRY: case ALEPH_GATE_CRZ:
    case ALEPH_GATE_UNITARY2Q: case ALEPH_GATE_UNITARY2QDIAG:
      return 2;
    case ALEPH_GATE_TOFFOLI: case ALEPH_GATE_CCZ: return 3;
    case ALEPH_GATE_UNITARYKQ: return g.k;
    default: return 1;
  }
}

// Gate::is_diagonal (kinds.rs:412-445)
bool is_diagonal(const PGate& g) {
  switch (g.kind) {
    case ALEPH_GATE_Z: case ALEPH_GATE_S: case ALEPH_GATE_SDG: case ALEPH_GATE_T: case ALEPH_GATE_TDG:
    case ALEPH_GATE_RZ: case ALEPH_GATE_PHASE: case ALEPH_GATE_CRZ: case ALEPH_GATE_CZ: case ALEPH_GATE_CCZ:
    case ALEPH_GATE_UNITARY1QDIAG: case ALEPH_GATE_UNITARY2QDIAG:
      return true;
    default: return false;
  }
}

// Gate::matrix (kinds.rs:213-400) through the oracle's restatement: the
// dense 2^a x 2^a matrix, or 0 on error (UnitaryKq has no fixed-size matrix).
int matrix(const PGate& g, C* out /* 64 */) {
  if (g.kind == ALEPH_GATE_UNITARYKQ) return 0;
  aleph_b200_instr r{};
  r.kind = g.kind;
  r.num_qubits = (uint32_t)g.q.size();
  for (size_t i = 0; i < g.q.size() && i < 8; ++i) r.qubits[i] = g.q[i];
  std::memcpy(r.params, g.p, sizeof(r.params));
  r.data_offset = 0;
  r.data_len = g.data.size();
  double buf[128];
  int dim = 0;
  if (orc_gate_matrix(&r, reinterpret_cast<const double*>(g.data.data()), g.data.size(), buf, &dim) != 0) return 0;
  for (int i = 0; i < dim * dim; ++i) out[i] = C(buf[2 * i], buf[2 * i + 1]);
  return dim;
}

bool matrix_ok(const PGate& g) {
  C m[64];
  return matrix(g, m) != 0;
}

std::vector<uint32_t> used_qubits(const PInst& in) {
  std::vector<uint32_t> out;
  switch (in.t) {
    case IK::Gate:
      out = in.g.q;
      out.insert(out.end(), in.g.c.begin(), in.g.c.end());
      break;
    case IK::Measure: case IK::Reset: out.push_back(in.qubit); break;
    case IK::Barrier: out = in.qs; break;
    case IK::Diag: {
      uint64_t m = 0;
      for (uint64_t c : in.conds) m |= c;
      for (uint32_t q = 0; q < in.dp_n && q < 64; ++q)
        if ((m >> q) & 1) out.push_back(q);
      break;
    }
    case IK::Tiled: {
      std::set<uint32_t> s;
      for (const PGate& g : in.gates) {
        s.insert(g.q.begin(), g.q.end());
        s.insert(g.c.begin(), g.c.end());
      }
      out.assign(s.begin(), s.end());
      break;
    }
  }
  return out;
}

// Gate::inverse (kinds.rs:506-555)
PGate inverse(const PGate& g) {
  PGate r = g;
  switch (g.kind) {
    case ALEPH_GATE_S: r.kind = ALEPH_GATE_SDG; break;
    case ALEPH_GATE_SDG: r.kind = ALEPH_GATE_S; break;
    case ALEPH_GATE_T: r.kind = ALEPH_GATE_TDG; break;
    case ALEPH_GATE_TDG: r.kind = ALEPH_GATE_T; break;
    case ALEPH_GATE_ISWAP: r.kind = ALEPH_GATE_ISWAPDG; break;
    case ALEPH_GATE_ISWAPDG: r.kind = ALEPH_GATE_ISWAP; break;
    case ALEPH_GATE_RX: case ALEPH_GATE_RY: case ALEPH_GATE_RZ: case ALEPH_GATE_PHASE:
    case ALEPH_GATE_CRX: case ALEPH_GATE_CRY: case ALEPH_GATE_CRZ:
      r.p[0] = -g.p[0];
      break;
    case ALEPH_GATE_U3:
      r.p[0] = -g.p[0];
      r.p[1] = -g.p[2];
      r.p[2] = -g.p[1];
      break;
    case ALEPH_GATE_UNITARY1Q: case ALEPH_GATE_UNITARY2Q: case ALEPH_GATE_UNITARYKQ: {
      const size_t dim = g.kind == ALEPH_GATE_UNITARY1Q ? 2 : g.kind == ALEPH_GATE_UNITARY2Q ? 4 : (size_t)1 << g.k;
      for (size_t i = 0; i < dim; ++i)
        for (size_t j = 0; j < dim; ++j) r.data[j * dim + i] = std::conj(g.data[i * dim + j]);
      break;
    }
    case ALEPH_GATE_UNITARY1QDIAG: case ALEPH_GATE_UNITARY2QDIAG:
      for (auto& z : r.data) z = std::conj(z);
      break;
    default: break;  // self-inverse
  }
  return r;
}

// `Gate` equality (derived PartialEq: kind, f64 parameters, matrix data)
bool same_gate(const PGate& a, const PGate& b) {
  if (a.kind != b.kind || a.k != b.k) return false;
  for (int i = 0; i < 3; ++i)
    if (!(a.p[i] == b.p[i])) return false;
  if (a.data.size() != b.data.size()) return false;
  for (size_t i = 0; i < a.data.size(); ++i)
    if (!(a.data[i].real() == b.data[i].real() && a.data[i].imag() == b.data[i].imag())) return false;
  return true;
}

PGate unitary1q(const C m[4], bool diag, uint32_t q) {
  PGate g;
  g.q = {q};
  if (diag) {
    g.kind = ALEPH_GATE_UNITARY1QDIAG;
    g.data = {m[0], m[3]};
  } else {
    g.kind = ALEPH_GATE_UNITARY1Q;
    g.data.assign(m, m + 4);
  }
  return g;
}

// ---- passes ------------------------------------------------------------------
struct PassCounts {
  uint64_t input, after_cancel, after_fuse1q, after_fuse2q, after_fusekq, output, tiled_blocks, fused_kq, relabeled;
};

// RelabelQubits::run (crates/aleph-ir/src/passes/relabel.rs:44-96) and
// count_confinable (relabel.rs:98-115)
size_t count_confinable(const std::vector<PInst>& v, uint32_t tb, const std::vector<uint32_t>* map) {
  size_t c = 0;
  for (const PInst& in : v) {
    if (in.t != IK::Gate || in.g.q.size() > 2 || !matrix_ok(in.g)) continue;
    bool all = true;
    for (uint32_t q : in.g.q) all = all && (map ? (*map)[q] : q) < tb;
    c += all;
  }
  return c;
}

void remap(PInst& in, const std::vector<uint32_t>& m) {
  switch (in.t) {
    case IK::Gate:
      for (auto& q : in.g.q) q = m[q];
      for (auto& q : in.g.c) q = m[q];
      break;
    case IK::Measure: case IK::Reset: in.qubit = m[in.qubit]; break;
    case IK::Barrier: for (auto& q : in.qs) q = m[q]; break;
    case IK::Diag:
      for (auto& cm : in.conds) {  // remap_diagonal_phase (relabel.rs:152-165)
        uint64_t out = 0, x = cm;
        while (x) {
          const int q = __builtin_ctzll(x);
          out |= 1ull << m[q];
          x &= x - 1;
        }
        cm = out;
      }
      break;
    case IK::Tiled: break;  // never present before TileBlock
  }
}

bool relabel_qubits(std::vector<PInst>& v, uint32_t n, uint32_t tile_bits, std::vector<uint32_t>* perm) {
  if (n <= 1) return false;
  std::vector<uint64_t> score(n, 0);
  for (const PInst& in : v)
    for (uint32_t q : used_qubits(in))
      if (q < n) ++score[q];
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return score[a] != score[b] ? score[a] > score[b] : a < b;
  });
  std::vector<uint32_t> phys(n);
  for (uint32_t b = 0; b < n; ++b) phys[order[b]] = b;
  if (count_confinable(v, tile_bits, &phys) <= count_confinable(v, tile_bits, nullptr)) return false;
  for (PInst& in : v) remap(in, phys);
  *perm = phys;
  return true;
}

// CancelInversePairs::run (crates/aleph-ir/src/passes/cancel.rs:35-137)
void cancel_inverse_pairs(std::vector<PInst>& v) {
  std::vector<PInst> result;
  std::vector<bool> removed;
  std::map<uint32_t, std::vector<size_t>> live;
  for (const PInst& in : v) {
    const std::vector<uint32_t> support = used_qubits(in);
    if (in.t != IK::Gate) {
      const size_t k = result.size();
      result.push_back(in);
      removed.push_back(false);
      for (uint32_t q : support) live[q].push_back(k);
      continue;
    }
    long cand = -1;
    bool shared = true;
    for (uint32_t q : support) {
      auto it = live.find(q);
      if (it == live.end() || it->second.empty()) {
        shared = false;
        break;
      }
      const long top = (long)it->second.back();
      if (cand < 0) cand = top;
      else if (cand != top) {
        shared = false;
        break;
      }
    }
    bool cancels = false;
    if (shared && cand >= 0 && result[cand].t == IK::Gate) {
      const PGate& prev = result[cand].g;
      std::vector<uint32_t> ca = prev.c, cb = in.g.c;
      std::sort(ca.begin(), ca.end());
      std::sort(cb.begin(), cb.end());
      cancels = prev.q == in.g.q && ca == cb && same_gate(prev, inverse(in.g));
    }
    if (cancels) {
      removed[cand] = true;
      for (uint32_t q : support) live[q].pop_back();
    } else {
      const size_t k = result.size();
      result.push_back(in);
      removed.push_back(false);
      for (uint32_t q : support) live[q].push_back(k);
    }
  }
  v.clear();
  for (size_t i = 0; i < result.size(); ++i)
    if (!removed[i]) v.push_back(std::move(result[i]));
}

void left_mul2(C acc[4], const C a[4]) {  // acc := a . acc
  const C b0 = acc[0], b1 = acc[1], b2 = acc[2], b3 = acc[3];
  acc[0] = a[0] * b0 + a[1] * b2;
  acc[1] = a[0] * b1 + a[1] * b3;
  acc[2] = a[2] * b0 + a[3] * b2;
  acc[3] = a[2] * b1 + a[3] * b3;
}

// Fuse1qRuns::run (crates/aleph-ir/src/passes/fuse_1q.rs:15-183)
void fuse_1q_runs(std::vector<PInst>& v) {
  struct Pending {
    size_t start;
    C m[4];
    bool diag;
    size_t len;
  };
  std::map<uint32_t, Pending> pending;
  std::vector<PInst> out;
  auto flush = [&](uint32_t q) {
    auto it = pending.find(q);
    if (it == pending.end()) return;
    const Pending& p = it->second;
    if (p.len == 1) out.push_back(v[p.start]);
    else {
      PInst in;
      in.t = IK::Gate;
      in.g = unitary1q(p.m, p.diag, q);
      out.push_back(std::move(in));
    }
    pending.erase(it);
  };
  for (size_t idx = 0; idx < v.size(); ++idx) {
    const PInst& in = v[idx];
    if (in.t == IK::Gate) {
      const PGate& g = in.g;
      if (arity(g) == 1 && g.c.empty() && g.q.size() == 1) {
        const uint32_t q = g.q[0];
        C m[64];
        if (matrix(g, m) != 2) {
          flush(q);
          out.push_back(in);
          continue;
        }
        auto it = pending.find(q);
        if (it != pending.end()) {
          left_mul2(it->second.m, m);
          it->second.diag = it->second.diag && is_diagonal(g);
          ++it->second.len;
        } else {
          Pending p{idx, {m[0], m[1], m[2], m[3]}, is_diagonal(g), 1};
          pending.emplace(q, p);
        }
        continue;
      }
    }
    for (uint32_t q : used_qubits(in)) flush(q);
    out.push_back(in);
  }
  std::vector<uint32_t> left;
  for (auto& kv : pending) left.push_back(kv.first);
  for (uint32_t q : left) flush(q);  // ascending qubit order
  v = std::move(out);
}

using M4 = std::array<C, 16>;

M4 mul4(const M4& a, const M4& b) {
  M4 o{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      C acc(0, 0);
      for (int k = 0; k < 4; ++k) acc += a[i * 4 + k] * b[k * 4 + j];
      o[i * 4 + j] = acc;
    }
  return o;
}
M4 ident4() {
  M4 m{};
  for (int i = 0; i < 4; ++i) m[i * 5] = 1.0;
  return m;
}
// lift_1q (fuse_2q.rs:52-77): m2 on q inside the block [hi, lo]
M4 lift_1q(const C m2[4], uint32_t q, uint32_t hi) {
  M4 o{};
  const bool on_high = q == hi;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      const int hr = (r >> 1) & 1, lr = r & 1, hc = (c >> 1) & 1, lc = c & 1;
      if (on_high) o[r * 4 + c] = lr == lc ? m2[hr * 2 + hc] : C(0, 0);
      else o[r * 4 + c] = hr == hc ? m2[lr * 2 + lc] : C(0, 0);
    }
  return o;
}
M4 reorder_swap(const M4& m) {  // fuse_2q.rs:81-92
  auto sw = [](int i) { return ((i & 1) << 1) | ((i >> 1) & 1); };
  M4 o{};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) o[r * 4 + c] = m[sw(r) * 4 + sw(c)];
  return o;
}

// Fuse2q::run (crates/aleph-ir/src/passes/fuse_2q.rs:97-480)
void fuse_2q(std::vector<PInst>& v) {
  struct Block {
    std::vector<uint32_t> q;  // [hi, lo] or [q]
    bool two;
    C m2[4];
    M4 m4;
    size_t first;
    size_t len;
    bool diag;
  };
  std::vector<Block> blocks;
  std::vector<bool> alive;
  std::map<uint32_t, size_t> open;
  std::vector<std::pair<size_t, PInst>> out;
  auto emit = [&](const Block& b) {
    if (b.len == 1) {
      out.emplace_back(b.first, v[b.first]);
      return;
    }
    PInst in;
    in.t = IK::Gate;
    if (!b.two) in.g = unitary1q(b.m2, b.diag, b.q[0]);
    else {
      in.g.kind = ALEPH_GATE_UNITARY2Q;
      in.g.q = b.q;
      in.g.data.assign(b.m4.begin(), b.m4.end());
    }
    out.emplace_back(b.first, std::move(in));
  };
  auto flush_block = [&](size_t id) {
    if (!alive[id]) return;
    alive[id] = false;
    for (uint32_t q : blocks[id].q) {
      auto it = open.find(q);
      if (it != open.end() && it->second == id) open.erase(it);
    }
    emit(blocks[id]);
  };
  auto flush_qubit = [&](uint32_t q) {
    auto it = open.find(q);
    if (it != open.end()) flush_block(it->second);
  };
  for (size_t idx = 0; idx < v.size(); ++idx) {
    const PInst& in = v[idx];
    if (in.t == IK::Gate && arity(in.g) == 1 && in.g.c.empty() && in.g.q.size() == 1) {
      const uint32_t q = in.g.q[0];
      C m[64];
      if (matrix(in.g, m) != 2) {
        flush_qubit(q);
        out.emplace_back(idx, in);
        continue;
      }
      auto it = open.find(q);
      if (it != open.end()) {
        Block& b = blocks[it->second];
        if (!b.two) {
          left_mul2(b.m2, m);
          b.diag = b.diag && is_diagonal(in.g);
        } else {
          b.m4 = mul4(lift_1q(m, q, b.q[0]), b.m4);
        }
        ++b.len;
      } else {
        Block b;
        b.q = {q};
        b.two = false;
        std::copy(m, m + 4, b.m2);
        b.first = idx;
        b.len = 1;
        b.diag = is_diagonal(in.g);
        blocks.push_back(b);
        alive.push_back(true);
        open[q] = blocks.size() - 1;
      }
      continue;
    }
    if (in.t == IK::Gate && arity(in.g) == 2 && in.g.c.empty() && in.g.q.size() == 2) {
      const uint32_t q0 = in.g.q[0], q1 = in.g.q[1];
      C mm[64];
      if (matrix(in.g, mm) != 4) {
        flush_qubit(q0);
        flush_qubit(q1);
        out.emplace_back(idx, in);
        continue;
      }
      M4 m4;
      std::copy(mm, mm + 16, m4.begin());
      auto a = open.find(q0), b = open.find(q1);
      if (a != open.end() && b != open.end() && a->second == b->second) {  // same-pair merge
        Block& bl = blocks[a->second];
        const M4 oriented = (bl.q[0] == q0 && bl.q[1] == q1) ? m4 : reorder_swap(m4);
        bl.m4 = mul4(oriented, bl.m4);
        ++bl.len;
        continue;
      }
      for (uint32_t q : {q0, q1}) {  // a 2q block cannot be a pre-1q
        auto it = open.find(q);
        if (it != open.end() && blocks[it->second].two) flush_block(it->second);
      }
      M4 pre = ident4();
      size_t len = 1;
      for (uint32_t q : {q0, q1}) {
        auto it = open.find(q);
        if (it != open.end()) {
          const size_t id = it->second;
          alive[id] = false;
          open.erase(it);
          pre = mul4(lift_1q(blocks[id].m2, q, q0), pre);
          len += blocks[id].len;
        }
      }
      Block nb;
      nb.q = {q0, q1};
      nb.two = true;
      nb.m4 = mul4(m4, pre);
      nb.first = idx;  // keyed at the 2q gate's own index (fuse_2q.rs:335-355)
      nb.len = len;
      nb.diag = false;
      blocks.push_back(nb);
      alive.push_back(true);
      open[q0] = blocks.size() - 1;
      open[q1] = blocks.size() - 1;
      continue;
    }
    for (uint32_t q : used_qubits(in)) flush_qubit(q);
    out.emplace_back(idx, in);
  }
  for (size_t id = 0; id < blocks.size(); ++id) flush_block(id);
  std::stable_sort(out.begin(), out.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  v.clear();
  for (auto& pr : out) v.push_back(std::move(pr.second));
}

// lift_dense (crates/aleph-ir/src/passes/fuse_kq.rs:49-100): a gate's dense
// matrix on MSB-first `gq` embedded in the block over ascending `bq`.
std::vector<C> lift_dense(const C* gd, const std::vector<uint32_t>& gq, const std::vector<uint32_t>& bq) {
  const size_t k = bq.size(), dim = (size_t)1 << k, ga = gq.size(), gdim = (size_t)1 << ga;
  std::vector<size_t> bb(ga);
  for (size_t a = 0; a < ga; ++a) bb[a] = k - 1 - (size_t)(std::find(bq.begin(), bq.end(), gq[a]) - bq.begin());
  std::vector<C> out(dim * dim, C(0, 0));
  for (size_t col = 0; col < dim; ++col) {
    size_t gin = 0;
    for (size_t a = 0; a < ga; ++a) gin |= ((col >> bb[a]) & 1) << (ga - 1 - a);
    for (size_t grow = 0; grow < gdim; ++grow) {
      const C amp = gd[grow * gdim + gin];
      if (amp == C(0, 0)) continue;
      size_t row = col;
      for (size_t a = 0; a < ga; ++a) {
        const size_t ob = (grow >> (ga - 1 - a)) & 1;
        row = (row & ~((size_t)1 << bb[a])) | (ob << bb[a]);
      }
      out[row * dim + col] += amp;
    }
  }
  return out;
}

std::vector<C> matmul(const std::vector<C>& a, const std::vector<C>& b, size_t n) {
  std::vector<C> o(n * n, C(0, 0));
  for (size_t i = 0; i < n; ++i)
    for (size_t k = 0; k < n; ++k) {
      const C aik = a[i * n + k];
      if (aik == C(0, 0)) continue;
      for (size_t j = 0; j < n; ++j) o[i * n + j] += aik * b[k * n + j];
    }
  return o;
}

// FuseKq::run (crates/aleph-ir/src/passes/fuse_kq.rs:255-400), build_block_matrix (:102-142)
void fuse_kq(std::vector<PInst>& v, uint32_t n, uint32_t max_qubits) {
  const uint32_t max_k = std::min<uint32_t>(5, std::max<uint32_t>(2, max_qubits));
  struct Block {
    std::set<uint32_t> q;
    std::vector<std::pair<size_t, PGate>> members;
    size_t first;
  };
  std::vector<Block> blocks;
  std::vector<bool> alive;
  std::vector<long> owner(n, -1);
  std::vector<PInst> out;
  auto close_block = [&](Block& b) {
    std::stable_sort(b.members.begin(), b.members.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    if (b.q.size() >= 3 && b.members.size() >= 2) {
      const std::vector<uint32_t> bq(b.q.begin(), b.q.end());
      const size_t dim = (size_t)1 << bq.size();
      std::vector<C> acc(dim * dim, C(0, 0));
      for (size_t i = 0; i < dim; ++i) acc[i * dim + i] = 1.0;
      for (auto& mb : b.members) {
        const PGate& g = mb.second;
        std::vector<C> lifted;
        C m[64];
        const int d = matrix(g, m);
        lifted = lift_dense(m, g.q, bq);
        (void)d;
        acc = matmul(lifted, acc, dim);
      }
      PInst in;
      in.t = IK::Gate;
      in.g.kind = ALEPH_GATE_UNITARYKQ;
      in.g.k = (uint32_t)bq.size();
      in.g.q = bq;
      in.g.data = std::move(acc);
      out.push_back(std::move(in));
    } else {
      for (auto& mb : b.members) {
        PInst in;
        in.t = IK::Gate;
        in.g = std::move(mb.second);
        out.push_back(std::move(in));
      }
    }
  };
  auto close_touching = [&](const std::vector<uint32_t>& qs) {
    std::set<long> ids;
    for (uint32_t q : qs)
      if (q < n && owner[q] >= 0) ids.insert(owner[q]);
    std::vector<long> ord(ids.begin(), ids.end());
    std::stable_sort(ord.begin(), ord.end(), [&](long a, long b) { return blocks[a].first < blocks[b].first; });
    for (long id : ord) {
      if (!alive[id]) continue;
      alive[id] = false;
      for (uint32_t q : blocks[id].q) owner[q] = -1;
      close_block(blocks[id]);
    }
  };
  for (size_t idx = 0; idx < v.size(); ++idx) {
    const PInst& in = v[idx];
    const bool fusable = in.t == IK::Gate && in.g.c.empty() && in.g.kind != ALEPH_GATE_UNITARYKQ && matrix_ok(in.g);
    if (!fusable) {
      close_touching(used_qubits(in));
      out.push_back(in);
      continue;
    }
    std::vector<uint32_t> support = in.g.q;
    std::sort(support.begin(), support.end());
    std::set<long> dep;
    for (uint32_t q : support)
      if (owner[q] >= 0) dep.insert(owner[q]);
    std::set<uint32_t> merged(support.begin(), support.end());
    for (long id : dep) merged.insert(blocks[id].q.begin(), blocks[id].q.end());
    if (merged.size() <= max_k) {
      Block nb;
      nb.first = idx;
      for (long id : dep) {
        alive[id] = false;
        nb.first = std::min(nb.first, blocks[id].first);
        for (auto& m : blocks[id].members) nb.members.push_back(std::move(m));
      }
      nb.members.emplace_back(idx, in.g);
      nb.q = merged;
      blocks.push_back(std::move(nb));
      alive.push_back(true);
      for (uint32_t q : merged) owner[q] = (long)blocks.size() - 1;
    } else {
      std::vector<uint32_t> dq;
      for (long id : dep) dq.insert(dq.end(), blocks[id].q.begin(), blocks[id].q.end());
      close_touching(dq);
      Block nb;
      nb.first = idx;
      nb.members.emplace_back(idx, in.g);
      nb.q = std::set<uint32_t>(support.begin(), support.end());
      blocks.push_back(std::move(nb));
      alive.push_back(true);
      for (uint32_t q : support) owner[q] = (long)blocks.size() - 1;
    }
  }
  std::vector<long> rem;
  for (size_t id = 0; id < blocks.size(); ++id)
    if (alive[id]) rem.push_back((long)id);
  std::stable_sort(rem.begin(), rem.end(), [&](long a, long b) { return blocks[a].first < blocks[b].first; });
  for (long id : rem) {
    alive[id] = false;
    close_block(blocks[id]);
  }
  v = std::move(out);
}

// ---- FuseDiagonalRuns (crates/aleph-ir/src/passes/fuse_diagonal.rs) ----------------
// GF(2) bit-permutation tracker (Perm, fuse_diagonal.rs:205-246): row[i] is the
// mask whose parity with the run-start basis gives current bit i.
struct GfPerm {
  std::vector<uint64_t> row;
  explicit GfPerm(uint32_t n) : row(n) {
    for (uint32_t i = 0; i < n; ++i) row[i] = 1ull << i;
  }
  void cx(uint32_t c, uint32_t t) { row[t] ^= row[c]; }
  uint64_t image(uint32_t b) const { return row[b]; }
  uint64_t image_of_mask(uint64_t m) const {
    uint64_t o = 0;
    for (; m; m &= m - 1) o ^= row[__builtin_ctzll(m)];
    return o;
  }
  bool identity() const {
    for (size_t i = 0; i < row.size(); ++i)
      if (row[i] != 1ull << i) return false;
    return true;
  }
};

constexpr double kPhaseEps = 1e-12;  // PHASE_EPS (fuse_diagonal.rs:249)

double rem_2pi(double a) {  // f64::rem_euclid(2 pi)
  const double tp = 2.0 * M_PI;
  const double r = std::fmod(a, tp);
  return r < 0 ? r + tp : r;
}

struct DTerm {
  std::vector<uint64_t> conds;
  double angle;
};

// diagonal_to_terms (fuse_diagonal.rs:266-310): the phase function of a
// diagonal gate as a multilinear polynomial over its targets (Moebius
// inversion), each monomial's conds mapped through the tracker; external
// controls condition every term.
bool diagonal_to_terms(const PGate& g, const GfPerm& perm, std::vector<DTerm>* out) {
  if (!is_diagonal(g)) return false;
  C m[64];
  const int dim = matrix(g, m);
  if (!dim) return false;
  const uint32_t k = (uint32_t)g.q.size();
  auto f = [&](uint32_t pattern) {
    uint32_t r = 0;
    for (uint32_t p = 0; p < k; ++p)
      if ((pattern >> p) & 1) r |= 1u << (k - 1 - p);
    return std::arg(m[r * dim + r]);
  };
  for (uint32_t s = 0; s < (1u << k); ++s) {
    double alpha = 0.0;
    for (uint32_t t = s;; t = (t - 1) & s) {
      alpha += ((__builtin_popcount(s ^ t) & 1) ? -1.0 : 1.0) * f(t);
      if (t == 0) break;
    }
    const double a = rem_2pi(alpha);
    if (a < kPhaseEps || 2.0 * M_PI - a < kPhaseEps) continue;
    DTerm term;
    for (uint32_t p = 0; p < k; ++p)
      if ((s >> p) & 1) term.conds.push_back(perm.image(g.q[p]));
    for (uint32_t c : g.c) term.conds.push_back(perm.image(c));
    term.angle = alpha;
    out->push_back(std::move(term));
  }
  return true;
}

bool diag_run_member(const PInst& in) {  // is_run_member (fuse_diagonal.rs:72-80)
  if (in.t == IK::Diag) return true;
  return in.t == IK::Gate && (is_diagonal(in.g) || (in.g.kind == ALEPH_GATE_CNOT && in.g.c.empty()));
}

// fuse_run (fuse_diagonal.rs:86-157) and canonicalize (:164-190): one
// DiagonalPhase for the run, or false to re-emit the run verbatim.
bool fuse_diag_run(const std::vector<PInst>& v, size_t i0, size_t i1, uint32_t n, PInst* out) {
  GfPerm perm(n);
  std::vector<DTerm> terms;
  size_t gates = 0;
  uint64_t support = 0;
  for (size_t i = i0; i < i1; ++i) {
    const PInst& in = v[i];
    if (in.t == IK::Diag) {
      if (in.dp_n != n) return false;
      for (uint64_t c : in.conds)
        if (n < 64 && (c >> n) != 0) return false;
      for (const aleph_b200_phase_term& t : in.terms) {
        DTerm d;
        for (uint32_t c = 0; c < t.cond_count; ++c) {
          d.conds.push_back(perm.image_of_mask(in.conds[t.cond_offset + c]));
          support |= d.conds.back();
        }
        d.angle = t.angle;
        terms.push_back(std::move(d));
      }
      ++gates;
      continue;
    }
    const PGate& g = in.g;
    if (g.kind == ALEPH_GATE_CNOT) {
      if (!g.c.empty() || g.q.size() < 2) return false;
      perm.cx(g.q[0], g.q[1]);
      support |= (1ull << g.q[0]) | (1ull << g.q[1]);
    } else {
      if (!diagonal_to_terms(g, perm, &terms)) return false;
      ++gates;
      for (uint32_t q : g.q) support |= 1ull << q;
      for (uint32_t c : g.c) support |= 1ull << c;
    }
  }
  if (!perm.identity()) return false;
  if (__builtin_popcountll(support) <= 1 || gates < 2) return false;
  // merge terms with the same (sorted) condition set, in key order
  std::map<std::vector<uint64_t>, double> merged;
  for (DTerm& t : terms) {
    std::sort(t.conds.begin(), t.conds.end());
    auto it = merged.find(t.conds);
    if (it == merged.end()) merged.emplace(t.conds, t.angle);
    else it->second += t.angle;
  }
  out->t = IK::Diag;
  out->dp_n = n;
  out->terms.clear();
  out->conds.clear();
  for (const auto& kv : merged) {
    const double a = rem_2pi(kv.second);
    if (a < kPhaseEps || 2.0 * M_PI - a < kPhaseEps) continue;
    aleph_b200_phase_term t;
    t.angle = kv.second;
    t.cond_offset = (uint32_t)out->conds.size();
    t.cond_count = (uint32_t)kv.first.size();
    out->conds.insert(out->conds.end(), kv.first.begin(), kv.first.end());
    out->terms.push_back(t);
  }
  return true;
}

// FuseDiagonalRuns::run (fuse_diagonal.rs:23-68): maximal runs of diagonal
// gates, bare CNOTs and DiagonalPhase records become one DiagonalPhase each.
void fuse_diagonal_runs(std::vector<PInst>& v, uint32_t n) {
  std::vector<PInst> out;
  size_t i = 0;
  while (i < v.size()) {
    if (!diag_run_member(v[i])) {
      out.push_back(std::move(v[i]));
      ++i;
      continue;
    }
    size_t j = i;
    while (j < v.size() && diag_run_member(v[j])) ++j;
    PInst dp;
    if (fuse_diag_run(v, i, j, n, &dp)) out.push_back(std::move(dp));
    else
      for (size_t k = i; k < j; ++k) out.push_back(std::move(v[k]));
    i = j;
  }
  v = std::move(out);
}

// TileBlock::run (crates/aleph-ir/src/passes/tile_block.rs:47-110)
void tile_block(std::vector<PInst>& v, uint32_t tile_bits) {
  std::vector<PInst> out;
  std::vector<PGate> run;
  auto flush = [&]() {
    if (run.size() == 1) {
      PInst in;
      in.t = IK::Gate;
      in.g = std::move(run[0]);
      out.push_back(std::move(in));
    } else if (run.size() > 1) {
      PInst in;
      in.t = IK::Tiled;
      in.gates = std::move(run);
      in.tile_bits = tile_bits;
      out.push_back(std::move(in));
    }
    run.clear();
  };
  for (PInst& in : v) {
    bool conf = in.t == IK::Gate && in.g.q.size() <= 2 && matrix_ok(in.g);
    if (conf)
      for (uint32_t q : in.g.q) conf = conf && q < tile_bits;
    if (conf) run.push_back(std::move(in.g));
    else {
      flush();
      out.push_back(std::move(in));
    }
  }
  flush();
  v = std::move(out);
}

// ---- CPU sv kernels (timing path) ------------------------------------------------
// Index of the i-th amplitude with zeros at the ascending bit positions `pos`.
inline uint64_t deposit(uint64_t i, const uint32_t* pos, int k) {
  for (int j = 0; j < k; ++j) {
    const uint64_t lo = i & ((1ull << pos[j]) - 1);
    i = ((i >> pos[j]) << (pos[j] + 1)) | lo;
  }
  return i;
}

// One dense gate on K targets: per outer index, gather the 2^K amplitudes,
// multiply by the matrix (held transposed, real and imaginary parts apart, so
// the row loop vectorises), scatter. The reference's unitary_kq /
// apply_2q_dense kernels (crates/aleph-sv/src/kernels/unitary_kq.rs:127-166,
// kernels/aos.rs:1335-1394) do the same gather / matvec / scatter.
template <int K>
void dense_k(C* a, int64_t outer, const uint32_t* pos, const uint64_t* off, const C* m, uint64_t cmask, bool par) {
  constexpr int D = 1 << K;
  alignas(64) double mr[D][D], mi[D][D];  // [c][r]
  for (int r = 0; r < D; ++r)
    for (int c = 0; c < D; ++c) {
      mr[c][r] = m[r * D + c].real();
      mi[c][r] = m[r * D + c].imag();
    }
  double* ad = reinterpret_cast<double*>(a);
  auto body = [&](int64_t i) {
    const uint64_t base = deposit((uint64_t)i, pos, K);
    if ((base & cmask) != cmask) return;
    double vr[D], vi[D], ar[D], ai[D];
    for (int c = 0; c < D; ++c) {
      vr[c] = ad[2 * (base | off[c])];
      vi[c] = ad[2 * (base | off[c]) + 1];
    }
    if constexpr (D >= 4) {
      // rows four at a time in AVX2 registers
      __m256d accr[D / 4], acci[D / 4];
      for (int r = 0; r < D / 4; ++r) accr[r] = acci[r] = _mm256_setzero_pd();
      for (int c = 0; c < D; ++c) {
        const __m256d xr = _mm256_set1_pd(vr[c]), xi = _mm256_set1_pd(vi[c]);
        for (int r = 0; r < D / 4; ++r) {
          const __m256d wr = _mm256_load_pd(&mr[c][4 * r]), wi = _mm256_load_pd(&mi[c][4 * r]);
          accr[r] = _mm256_fnmadd_pd(wi, xi, _mm256_fmadd_pd(wr, xr, accr[r]));
          acci[r] = _mm256_fmadd_pd(wi, xr, _mm256_fmadd_pd(wr, xi, acci[r]));
        }
      }
      for (int r = 0; r < D / 4; ++r) {
        _mm256_storeu_pd(&ar[4 * r], accr[r]);
        _mm256_storeu_pd(&ai[4 * r], acci[r]);
      }
    } else {
      for (int r = 0; r < D; ++r) ar[r] = ai[r] = 0.0;
      for (int c = 0; c < D; ++c) {
        const double xr = vr[c], xi = vi[c];
        for (int r = 0; r < D; ++r) {
          ar[r] += mr[c][r] * xr - mi[c][r] * xi;
          ai[r] += mr[c][r] * xi + mi[c][r] * xr;
        }
      }
    }
    for (int r = 0; r < D; ++r) {
      ad[2 * (base | off[r])] = ar[r];
      ad[2 * (base | off[r]) + 1] = ai[r];
    }
  };
  if (par) {
#pragma omp parallel for schedule(static) num_threads(threads())
    for (int64_t i = 0; i < outer; ++i) body(i);
  } else {
    for (int64_t i = 0; i < outer; ++i) body(i);
  }
}

// One dense gate (k targets, MSB-first operands) with controls, over amplitudes
// a[0 .. 2^n). `par`: OpenMP over the outer index (whole-state gates); a tile
// of a TiledBlock runs it serially inside its own task. Diagonal matrices take
// the phase-multiply path (the reference's diagonal classifiers,
// crates/aleph-sv/src/kernels/mod.rs:358-486).
void apply_dense(C* a, uint32_t n, const std::vector<uint32_t>& t, const C* m, uint64_t cmask, bool par) {
  const int k = std::min<int>((int)t.size(), 5);  // prepare() admits at most 5 targets
  const uint64_t dim = 1ull << k;
  uint32_t pos[8];
  for (int j = 0; j < k; ++j) pos[j] = t[j];
  std::sort(pos, pos + k);
  uint64_t off[32];
  for (uint64_t r = 0; r < dim; ++r) {
    uint64_t o = 0;
    for (int p = 0; p < k; ++p)
      if ((r >> p) & 1) o |= 1ull << t[k - 1 - p];
    off[r] = o;
  }
  bool diag = true;
  for (uint64_t r = 0; r < dim && diag; ++r)
    for (uint64_t c = 0; c < dim; ++c)
      if (r != c && m[r * dim + c] != C(0, 0)) {
        diag = false;
        break;
      }
  const int64_t outer = (int64_t)1 << (n - k);
  if (diag) {
    C d[32];
    for (uint64_t r = 0; r < dim; ++r) d[r] = m[r * dim + r];
    auto body = [&](int64_t i) {
      const uint64_t base = deposit((uint64_t)i, pos, k);
      if ((base & cmask) != cmask) return;
      for (uint64_t r = 0; r < dim; ++r) {
        C& x = a[base | off[r]];
        const double xr = x.real(), xi = x.imag();
        x = C(xr * d[r].real() - xi * d[r].imag(), xr * d[r].imag() + xi * d[r].real());
      }
    };
    if (par) {
#pragma omp parallel for schedule(static) num_threads(threads())
      for (int64_t i = 0; i < outer; ++i) body(i);
    } else {
      for (int64_t i = 0; i < outer; ++i) body(i);
    }
    return;
  }
  switch (k) {
    case 1: dense_k<1>(a, outer, pos, off, m, cmask, par); break;
    case 2: dense_k<2>(a, outer, pos, off, m, cmask, par); break;
    case 3: dense_k<3>(a, outer, pos, off, m, cmask, par); break;
    case 4: dense_k<4>(a, outer, pos, off, m, cmask, par); break;
    default: dense_k<5>(a, outer, pos, off, m, cmask, par); break;
  }
}

struct Ready {
  std::vector<uint32_t> t;
  std::vector<C> m;
  uint64_t cmask = 0;
  std::vector<uint32_t> controls;
};

int prepare(const PGate& g, uint32_t n, Ready* r) {
  if (g.kind == ALEPH_GATE_UNITARYKQ) r->m = g.data;
  else {
    C m[64];
    const int dim = matrix(g, m);
    if (!dim) return ALEPH_B200_UNSUPPORTED_GATE;
    r->m.assign(m, m + dim * dim);
  }
  if (g.q.empty() || g.q.size() > 5) return ALEPH_B200_UNSUPPORTED_GATE;
  r->t = g.q;
  r->controls = g.c;
  for (uint32_t q : g.q)
    if (q >= n) return ALEPH_B200_QUBIT_OUT_OF_RANGE;
  for (uint32_t c : g.c) {
    if (c >= n) return ALEPH_B200_QUBIT_OUT_OF_RANGE;
    r->cmask |= 1ull << c;
  }
  return ALEPH_B200_OK;
}

// NaiveSvBackend::apply_tiled_block (crates/aleph-sv/src/backend.rs:173-208) and
// apply_gate_to_tile (:231-253): tiles of 2^t amplitudes in parallel, every
// gate of the block applied to a tile before the next tile; a control at or
// above t is constant over a tile and skips it when 0.
int apply_tiled(C* a, uint32_t n, const PInst& in) {
  std::vector<Ready> rs(in.gates.size());
  for (size_t i = 0; i < in.gates.size(); ++i) {
    if (in.gates[i].q.size() > 2) return ALEPH_B200_UNSUPPORTED_GATE;
    if (int s = prepare(in.gates[i], n, &rs[i])) return s;
  }
  const uint32_t t = in.tile_bits;
  if (t >= n) {
    for (const Ready& r : rs) apply_dense(a, n, r.t, r.m.data(), r.cmask, true);
    return ALEPH_B200_OK;
  }
  const int64_t tiles = (int64_t)1 << (n - t);
#pragma omp parallel for schedule(static) num_threads(threads())
  for (int64_t tile = 0; tile < tiles; ++tile) {
    const uint64_t tb = (uint64_t)tile << t;
    C* base = a + tb;
    for (const Ready& r : rs) {
      uint64_t low = 0;
      bool skip = false;
      for (uint32_t c : r.controls) {
        if (c >= t) skip = skip || ((tb >> c) & 1) == 0;
        else low |= 1ull << c;
      }
      if (!skip) apply_dense(base, t, r.t, r.m.data(), low, false);
    }
  }
  return ALEPH_B200_OK;
}

// ---- the flat record stream -------------------------------------------------------
int parse(const aleph_b200_instr* in, uint64_t count, const aleph_b200_pools* pools, std::vector<PInst>* out) {
  const double* pool = pools ? pools->matrix_pool : nullptr;
  const uint64_t pool_len = pools ? pools->matrix_pool_len : 0;
  auto gate = [&](const aleph_b200_instr& r, PGate* g) {
    g->kind = r.kind;
    g->q.assign(r.qubits, r.qubits + std::min<uint32_t>(r.num_qubits, 8));
    g->c.assign(r.controls, r.controls + std::min<uint32_t>(r.num_controls, 8));
    std::memcpy(g->p, r.params, sizeof(g->p));
    g->k = r.kind == ALEPH_GATE_UNITARYKQ ? r.aux : 0;
    if (is_unitary_kind(r.kind)) {
      if (!pool || r.data_offset + r.data_len > pool_len) return false;
      const C* d = reinterpret_cast<const C*>(pool) + r.data_offset;
      g->data.assign(d, d + r.data_len);
    }
    return true;
  };
  for (uint64_t i = 0; i < count; ++i) {
    const aleph_b200_instr& r = in[i];
    PInst p;
    if (r.kind < 28) {
      p.t = IK::Gate;
      if (!gate(r, &p.g)) return ALEPH_B200_INVALID_ARGUMENT;
    } else if (r.kind == ALEPH_INSTR_MEASURE) {
      p.t = IK::Measure;
      p.qubit = r.qubits[0];
      p.clbit = r.aux;
    } else if (r.kind == ALEPH_INSTR_RESET) {
      p.t = IK::Reset;
      p.qubit = r.qubits[0];
    } else if (r.kind == ALEPH_INSTR_BARRIER) {
      p.t = IK::Barrier;  // its qubits as a mask in data_offset
      for (uint32_t q = 0; q < 64; ++q)
        if ((r.data_offset >> q) & 1) p.qs.push_back(q);
    } else if (r.kind == ALEPH_INSTR_DIAGONAL_PHASE) {
      p.t = IK::Diag;
      p.dp_n = r.aux;
      if (!pools || r.data_offset + r.data_len > pools->n_terms) return ALEPH_B200_INVALID_ARGUMENT;
      for (uint64_t k = 0; k < r.data_len; ++k) {
        aleph_b200_phase_term t = pools->terms[r.data_offset + k];
        if ((uint64_t)t.cond_offset + t.cond_count > pools->n_conds) return ALEPH_B200_INVALID_ARGUMENT;
        const uint32_t off = (uint32_t)p.conds.size();
        for (uint32_t c = 0; c < t.cond_count; ++c) p.conds.push_back(pools->cond_pool[t.cond_offset + c]);
        t.cond_offset = off;
        p.terms.push_back(t);
      }
    } else if (r.kind == ALEPH_INSTR_TILED_BLOCK) {
      p.t = IK::Tiled;
      p.tile_bits = r.aux;
      if (r.data_len > count - i - 1) return ALEPH_B200_INVALID_ARGUMENT;
      for (uint64_t k = 0; k < r.data_len; ++k) {
        PGate g;
        if (in[i + 1 + k].kind >= 28 || !gate(in[i + 1 + k], &g)) return ALEPH_B200_INVALID_ARGUMENT;
        p.gates.push_back(std::move(g));
      }
      i += r.data_len;
    } else {
      return ALEPH_B200_UNSUPPORTED_INSTRUCTION;
    }
    out->push_back(std::move(p));
  }
  return ALEPH_B200_OK;
}

void plan(std::vector<PInst>& v, uint32_t n, uint32_t tile_bits, uint32_t max_k, std::vector<uint32_t>* perm,
          PassCounts* pc) {
  pc->input = v.size();
  pc->relabeled = relabel_qubits(v, n, tile_bits, perm);
  cancel_inverse_pairs(v);
  pc->after_cancel = v.size();
  fuse_1q_runs(v);
  pc->after_fuse1q = v.size();
  fuse_2q(v);
  pc->after_fuse2q = v.size();
  fuse_kq(v, n, max_k);
  pc->after_fusekq = v.size();
  tile_block(v, tile_bits);
  pc->output = v.size();
  pc->tiled_blocks = 0;
  pc->fused_kq = 0;
  for (const PInst& in : v) {
    pc->tiled_blocks += in.t == IK::Tiled;
    pc->fused_kq += in.t == IK::Gate && in.g.kind == ALEPH_GATE_UNITARYKQ;
  }
}

// fuse_full_state (crates/aleph-cuda/src/fusion.rs:137-152), the pass list of
// the reference's CUDA execution plan (CudaExecutionPlan::compile,
// crates/aleph-cuda/src/execution.rs:118-126): CancelInversePairs,
// FuseDiagonalRuns, Fuse1qRuns, Fuse2q, FuseKq (width MAX_FUSE_QUBITS = 3). No
// relabelling and no tiling. pc->tiled_blocks counts the DiagonalPhase records.
void plan_gpu(std::vector<PInst>& v, uint32_t n, uint32_t max_k, PassCounts* pc) {
  pc->input = v.size();
  pc->relabeled = 0;
  cancel_inverse_pairs(v);
  pc->after_cancel = v.size();
  fuse_diagonal_runs(v, n);
  fuse_1q_runs(v);
  pc->after_fuse1q = v.size();
  fuse_2q(v);
  pc->after_fuse2q = v.size();
  fuse_kq(v, n, max_k);
  pc->after_fusekq = v.size();
  pc->output = v.size();
  pc->tiled_blocks = 0;
  pc->fused_kq = 0;
  for (const PInst& in : v) {
    pc->tiled_blocks += in.t == IK::Diag;
    pc->fused_kq += in.t == IK::Gate && in.g.kind == ALEPH_GATE_UNITARYKQ;
  }
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

/* Pass statistics of the pipeline on a record stream (host only):
 * out[0..9) = input, after CancelInversePairs, after Fuse1qRuns, after Fuse2q,
 * after FuseKq, output instructions, TiledBlocks, UnitaryKq blocks, relabelled. */
int orc_pipeline_describe(uint32_t n, const aleph_b200_instr* instrs, uint64_t count, const aleph_b200_pools* pools,
                          uint32_t tile_bits, uint32_t max_k, uint64_t* out) {
  std::vector<PInst> v;
  if (int s = parse(instrs, count, pools, &v)) return s;
  std::vector<uint32_t> perm;
  PassCounts pc{};
  plan(v, n, tile_bits, max_k, &perm, &pc);
  const uint64_t o[9] = {pc.input, pc.after_cancel, pc.after_fuse1q, pc.after_fuse2q, pc.after_fusekq,
                         pc.output, pc.tiled_blocks, pc.fused_kq, pc.relabeled};
  std::memcpy(out, o, sizeof(o));
  return ALEPH_B200_OK;
}

/* A planned circuit: the optimised instruction list of the final-state CPU
 * pipeline and its qubit permutation, executed by orc_pipeline_exec. */
struct orc_pipeline {
  std::vector<PInst> v;
  std::vector<uint32_t> perm;
  PassCounts pc{};
  uint32_t n = 0;
  double plan_s = 0;
  // the planned list as flat records (orc_pipeline_records)
  std::vector<aleph_b200_instr> rec;
  std::vector<double> mpool;
  std::vector<aleph_b200_phase_term> tpool;
  std::vector<uint64_t> cpool;
};

/* The reference's CUDA pass list (fuse_full_state) on a record stream; the
 * result runs on the CPU through orc_pipeline_exec or is exported as records
 * for the GPU reference arm (ref_gpu.cpp). */
int orc_gpu_pipeline_plan(uint32_t n, const aleph_b200_instr* instrs, uint64_t count, const aleph_b200_pools* pools,
                          uint32_t max_k, orc_pipeline** out) {
  const double t0 = now();
  auto* P = new orc_pipeline();
  P->n = n;
  if (int s = parse(instrs, count, pools, &P->v)) {
    delete P;
    return s;
  }
  plan_gpu(P->v, n, max_k, &P->pc);
  P->plan_s = now() - t0;
  *out = P;
  return ALEPH_B200_OK;
}

/* The planned instructions as flat records and pools (owned by the plan).
 * Gates carry their matrix (Unitary*, UnitaryKq) in the matrix pool. */
int orc_pipeline_records(orc_pipeline* P, const aleph_b200_instr** instrs, uint64_t* count, aleph_b200_pools* pools) {
  P->rec.clear();
  P->mpool.clear();
  P->tpool.clear();
  P->cpool.clear();
  for (const PInst& in : P->v) {
    aleph_b200_instr r{};
    switch (in.t) {
      case IK::Gate: {
        const PGate& g = in.g;
        r.kind = g.kind;
        r.num_qubits = (uint32_t)std::min<size_t>(g.q.size(), 8);
        r.num_controls = (uint32_t)std::min<size_t>(g.c.size(), 8);
        for (uint32_t i = 0; i < r.num_qubits; ++i) r.qubits[i] = g.q[i];
        for (uint32_t i = 0; i < r.num_controls; ++i) r.controls[i] = g.c[i];
        std::memcpy(r.params, g.p, sizeof(r.params));
        r.aux = g.k;
        r.data_offset = P->mpool.size() / 2;
        r.data_len = g.data.size();
        for (const C& z : g.data) {
          P->mpool.push_back(z.real());
          P->mpool.push_back(z.imag());
        }
        break;
      }
      case IK::Diag:
        r.kind = ALEPH_INSTR_DIAGONAL_PHASE;
        r.aux = in.dp_n;
        r.data_offset = P->tpool.size();
        r.data_len = in.terms.size();
        for (aleph_b200_phase_term t : in.terms) {
          t.cond_offset += (uint32_t)P->cpool.size();
          P->tpool.push_back(t);
        }
        P->cpool.insert(P->cpool.end(), in.conds.begin(), in.conds.end());
        break;
      case IK::Measure:
        r.kind = ALEPH_INSTR_MEASURE;
        r.num_qubits = 1;
        r.qubits[0] = in.qubit;
        r.aux = in.clbit;
        break;
      case IK::Barrier:
        r.kind = ALEPH_INSTR_BARRIER;
        for (uint32_t q : in.qs) r.data_offset |= 1ull << q;
        break;
      default:
        return ALEPH_B200_UNSUPPORTED_INSTRUCTION;
    }
    P->rec.push_back(r);
  }
  *instrs = P->rec.data();
  *count = P->rec.size();
  pools->matrix_pool = P->mpool.data();
  pools->matrix_pool_len = P->mpool.size() / 2;
  pools->terms = P->tpool.data();
  pools->n_terms = P->tpool.size();
  pools->cond_pool = P->cpool.data();
  pools->n_conds = P->cpool.size();
  return ALEPH_B200_OK;
}

/* Pass counts of a plan (the layout of orc_pipeline_describe's output). */
void orc_pipeline_counts(const orc_pipeline* P, uint64_t* out) {
  const PassCounts& pc = P->pc;
  const uint64_t o[9] = {pc.input, pc.after_cancel, pc.after_fuse1q, pc.after_fuse2q, pc.after_fusekq,
                         pc.output, pc.tiled_blocks, pc.fused_kq, pc.relabeled};
  std::memcpy(out, o, sizeof(o));
}

int orc_pipeline_plan(uint32_t n, const aleph_b200_instr* instrs, uint64_t count, const aleph_b200_pools* pools,
                      uint32_t tile_bits, uint32_t max_k, orc_pipeline** out) {
  const double t0 = now();
  auto* P = new orc_pipeline();
  P->n = n;
  if (int s = parse(instrs, count, pools, &P->v)) {
    delete P;
    return s;
  }
  plan(P->v, n, tile_bits, max_k, &P->perm, &P->pc);
  P->plan_s = now() - t0;
  *out = P;
  return ALEPH_B200_OK;
}

uint64_t orc_pipeline_len(const orc_pipeline* P) { return P->v.size(); }

void orc_pipeline_free(orc_pipeline* P) { delete P; }

/* Executes planned instructions [i0, i1) on amps (2^n complex); `finish`
 * applies the final unpermute of a relabelled plan. Measurements take one
 * uniform each when both branches are non-degenerate, as orc_run_stream;
 * *used counts them. *seconds = wall time of the call. */
int orc_pipeline_exec(const orc_pipeline* P, double* amps_d, uint64_t i0, uint64_t i1, int finish,
                      const double* uniforms, uint64_t n_uniforms, uint64_t* used, double* seconds) {
  const double t0 = now();
  const uint32_t n = P->n;
  C* a = reinterpret_cast<C*>(amps_d);
  uint64_t u_used = used ? *used : 0;
  for (uint64_t i = i0; i < i1 && i < P->v.size(); ++i) {
    const PInst& in = P->v[i];
    switch (in.t) {
      case IK::Gate: {
        Ready r;
        if (int s = prepare(in.g, n, &r)) return s;
        apply_dense(a, n, r.t, r.m.data(), r.cmask, true);
        break;
      }
      case IK::Tiled:
        if (int s = apply_tiled(a, n, in)) return s;
        break;
      case IK::Diag:
        if (int s = orc_apply_diagonal_phase(amps_d, n, in.terms.data(), in.terms.size(), in.conds.data(),
                                             in.conds.size()))
          return s;
        break;
      case IK::Measure: {
        int outcome = 0, consumed = 0;
        const double u = u_used < n_uniforms ? uniforms[u_used] : NAN;
        if (int s = orc_measure(amps_d, n, in.qubit, u, &outcome, &consumed)) return s;
        u_used += consumed;
        break;
      }
      case IK::Barrier: break;
      case IK::Reset: return ALEPH_B200_UNSUPPORTED_INSTRUCTION;
    }
  }
  if (finish && P->pc.relabeled)
    if (int s = orc_unpermute(amps_d, n, P->perm.data())) return s;
  if (used) *used = u_used;
  if (seconds) *seconds = now() - t0;
  return ALEPH_B200_OK;
}

/* run_optimized_cpu_final_state (crates/aleph-backend/src/lib.rs:308-318) on
 * `amps` (2^n complex, initialised by the caller): plans the stream with the
 * final-state CPU pipeline, executes it, unpermutes.
 * seconds[0] = planning, seconds[1] = execution (incl. the unpermute). */
int orc_pipeline_run(double* amps_d, uint32_t n, const aleph_b200_instr* instrs, uint64_t count,
                     const aleph_b200_pools* pools, uint32_t tile_bits, uint32_t max_k, const double* uniforms,
                     uint64_t n_uniforms, double* seconds, uint64_t* counts_out) {
  orc_pipeline* P = nullptr;
  if (int s = orc_pipeline_plan(n, instrs, count, pools, tile_bits, max_k, &P)) return s;
  uint64_t used = 0;
  double ex = 0;
  const int s = orc_pipeline_exec(P, amps_d, 0, P->v.size(), 1, uniforms, n_uniforms, &used, &ex);
  if (s == ALEPH_B200_OK) {
    if (seconds) {
      seconds[0] = P->plan_s;
      seconds[1] = ex;
    }
    if (counts_out) {
      const PassCounts& pc = P->pc;
      const uint64_t o[9] = {pc.input, pc.after_cancel, pc.after_fuse1q, pc.after_fuse2q, pc.after_fusekq,
                             pc.output, pc.tiled_blocks, pc.fused_kq, pc.relabeled};
      std::memcpy(counts_out, o, sizeof(o));
    }
  }
  delete P;
  return s;
}

}  // extern "C"
