// api.cpp — the C ABI of the B200 state-vector engine (include/aleph_b200.h).
//
// Host orchestration only: validation and lowering (planner.cpp), one
// upload of the plan tables per call, stream-ordered kernel launches, and a
// single synchronisation where a value must come back to the caller. There
// is no host compute path: every amplitude update and every reduction runs
// in the CUDA kernels of this library.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <unordered_map>
#include <vector>

#include "engine.h"

using namespace ab;

struct aleph_b200_handle : Handle {};
struct aleph_b200_state : State {};

namespace {

// ---- per-handle RNG: xoshiro256** seeded through splitmix64 -----------------
// It supplies the variates of aleph_b200_measure (u < 0) and
// aleph_b200_sample_seeded. Explicit variates can always be passed instead,
// which is how outcome parity with the reference is established.
uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct HandleExt {
  uint64_t rng[4];
};
HandleExt* ext(aleph_b200_handle* h);

uint64_t rng_next(aleph_b200_handle* h) {
  uint64_t* s = ext(h)->rng;
  const uint64_t result = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}
double rng_f64(aleph_b200_handle* h) { return (double)(rng_next(h) >> 11) * (1.0 / 9007199254740992.0); }

struct FullHandle : aleph_b200_handle {
  HandleExt x;
};
HandleExt* ext(aleph_b200_handle* h) { return &static_cast<FullHandle*>(h)->x; }

// ---- errors -----------------------------------------------------------------
int set_error(aleph_b200_handle* h, int status, const char* fmt, ...) {
  if (!h) return status;
  h->err.status = status;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  h->err_msg = buf;
  return status;
}

// Display strings of BackendError (crates/aleph-backend/src/lib.rs:22-74).
int report(aleph_b200_handle* h, const aleph_b200_error_info& e) {
  h->err = e;
  switch (e.status) {
    case ALEPH_B200_OK: h->err_msg.clear(); return 0;
    case ALEPH_B200_QUBIT_OUT_OF_RANGE:
      return set_error(h, e.status, "qubit %u out of range for %u-qubit state", e.qubit, e.num_qubits);
    case ALEPH_B200_DUPLICATE_QUBIT: return set_error(h, e.status, "duplicate qubit %u in gate or query", e.qubit);
    case ALEPH_B200_ARITY_MISMATCH:
      return set_error(h, e.status, "gate `%s` expects %u qubits, got %u", e.kind, e.expected, e.got);
    case ALEPH_B200_UNSUPPORTED_GATE: return set_error(h, e.status, "gate `%s` is not supported by this backend", e.kind);
    case ALEPH_B200_UNSUPPORTED_INSTRUCTION:
      return set_error(h, e.status, "IR instruction `%s` is not supported by this backend", e.kind);
    case ALEPH_B200_NON_FINITE_PARAM:
      return set_error(h, e.status, "gate `%s` has a non-finite (NaN or infinite) parameter", e.kind);
    case ALEPH_B200_NON_UNITARY_MATRIX:
      return set_error(h, e.status, "user-supplied matrix is not unitary (max deviation = %e)", e.value);
    case ALEPH_B200_DEGENERATE_MEASUREMENT:
      return set_error(h, e.status, "measurement of qubit %u on degenerate branch (p = %e)", e.qubit, e.value);
    case ALEPH_B200_TOO_MANY_QUBITS:
      return set_error(h, e.status, "requested %u qubits exceeds backend limit of %u", e.requested, e.limit);
    case ALEPH_B200_INVALID_PAULI_STRING:
      return set_error(h, e.status, "Pauli string violates its invariants: %s", e.kind);
    case ALEPH_B200_INVALID_STATE: return set_error(h, e.status, "backend state is invalid: %s", e.kind);
    case ALEPH_B200_EMPTY_CIRCUIT: return set_error(h, e.status, "cannot run an empty circuit");
    default: return set_error(h, e.status, "%s", e.kind[0] ? e.kind : "invalid argument");
  }
}

int cuda_fail(aleph_b200_handle* h, cudaError_t err, const char* what) {
  h->err = aleph_b200_error_info{};
  h->err.status = ALEPH_B200_DEVICE_FAILURE;
  return set_error(h, ALEPH_B200_DEVICE_FAILURE, "device operation failed: %s: %s", what, cudaGetErrorString(err));
}

#define CK(expr, what)                                   \
  do {                                                   \
    cudaError_t _e = (expr);                             \
    if (_e != cudaSuccess) return cuda_fail(h, _e, what); \
  } while (0)
// CK that first runs a cleanup callable on the status it returns
#define CK_OR(expr, cleanup, what)                                 \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) return cleanup(cuda_fail(h, _e, what)); \
  } while (0)

int ensure(aleph_b200_handle* h, Scratch& s, size_t bytes) {
  if (s.bytes >= bytes) return 0;
  if (s.ptr) {
    cudaStreamSynchronize(h->stream);
    cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
  }
  size_t want = bytes < 4096 ? 4096 : bytes;
  cudaError_t e = cudaMalloc(&s.ptr, want);
  if (e != cudaSuccess) {
    s.ptr = nullptr;
    return cuda_fail(h, e, "scratch allocation");
  }
  s.bytes = want;
  return 0;
}

// Every host<->device copy of the engine goes through here so that the
// stats count the bytes that cross PCIe/C2C.
cudaError_t copy_async(aleph_b200_handle* h, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                       cudaStream_t s) {
  if (kind == cudaMemcpyHostToDevice) h->stats.h2d_bytes += bytes;
  if (kind == cudaMemcpyDeviceToHost) h->stats.d2h_bytes += bytes;
  return cudaMemcpyAsync(dst, src, bytes, kind, s);
}

int bind(aleph_b200_handle* h) {
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  return 0;
}

// ---- plan upload + execution --------------------------------------------------
struct DevPlan {
  Op* ops;
  void* coef;
  PolyTables poly;
  double* uniforms;
  int32_t* status;
  uint8_t* outcomes;
};

size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

// Runs a plan on a state. With `cache` (a compiled plan's own device buffer),
// the plan tables are uploaded once and later calls only refresh the per-call
// region (measurement variates, status words, outcomes).
int execute(aleph_b200_handle* h, aleph_b200_state* st, const Plan& P, const double* uniforms, uint32_t n_uniforms,
            std::vector<int32_t>* status_out, std::vector<uint8_t>* outcomes_out, Scratch* cache = nullptr,
            bool* cache_ready = nullptr) {
  const bool f64 = st->precision == ALEPH_B200_F64;
  Scratch& buf = cache ? *cache : h->plan_buf;
  const bool reuse = cache && cache_ready && *cache_ready;
  if (cache && n_uniforms > P.n_measures) n_uniforms = P.n_measures;  // at most one variate per measurement
  const uint32_t ucap = cache ? P.n_measures : n_uniforms;
  // host image of the device tables
  std::vector<float> coef32;
  if (!f64 && !reuse) {
    coef32.resize(P.coef.size());
    for (size_t i = 0; i < P.coef.size(); ++i) coef32[i] = (float)P.coef[i];
  }
  const size_t b_ops = al(P.ops.size() * sizeof(Op));
  const size_t b_coef = al(P.coef.size() * (f64 ? 8 : 4));
  const size_t b_pa = al(P.poly_angle.size() * 8), b_po = al(P.poly_off.size() * 4), b_pc = al(P.poly_cnt.size() * 4),
               b_pd = al(P.poly_conds.size() * 8);
  const size_t b_u = al((size_t)ucap * 8), b_s = al(64), b_o = al(P.n_measures + 1);
  const size_t b_img = al(P.block_images.size());
  const size_t total = b_img + b_ops + b_coef + b_pa + b_po + b_pc + b_pd + b_u + b_s + b_o;
  if (int r = ensure(h, buf, total)) return r;
  std::vector<uint8_t> img(reuse ? 0 : total, 0);
  size_t off = 0;
  auto put = [&](const void* src, size_t bytes, size_t span) -> size_t {
    const size_t at = off;
    if (bytes && !reuse) std::memcpy(img.data() + off, src, bytes);
    off += span;
    return at;
  };
  const size_t o_img = put(P.block_images.data(), P.block_images.size(), b_img);
  const size_t o_ops = put(P.ops.data(), P.ops.size() * sizeof(Op), b_ops);
  const size_t o_coef = f64 ? put(P.coef.data(), P.coef.size() * 8, b_coef) : put(coef32.data(), P.coef.size() * 4, b_coef);
  const size_t o_pa = put(P.poly_angle.data(), P.poly_angle.size() * 8, b_pa);
  const size_t o_po = put(P.poly_off.data(), P.poly_off.size() * 4, b_po);
  const size_t o_pc = put(P.poly_cnt.data(), P.poly_cnt.size() * 4, b_pc);
  const size_t o_pd = put(P.poly_conds.data(), P.poly_conds.size() * 8, b_pd);
  const size_t o_u = put(uniforms, (size_t)n_uniforms * 8, b_u);
  const size_t o_s = put(nullptr, 0, b_s);
  const size_t o_o = put(nullptr, 0, b_o);
  char* base = (char*)buf.ptr;
  if (!reuse) {
    CK(copy_async(h, buf.ptr, img.data(), total, cudaMemcpyHostToDevice, h->stream), "plan upload");
  } else {
    if (n_uniforms)
      CK(copy_async(h, base + o_u, uniforms, (size_t)n_uniforms * 8, cudaMemcpyHostToDevice, h->stream),
         "variates upload");
    CK(cudaMemsetAsync(base + o_s, 0, b_s + b_o, h->stream), "status clear");
  }
  if (cache_ready) *cache_ready = true;
  DevPlan d;
  d.ops = (Op*)(base + o_ops);
  d.coef = base + o_coef;
  d.poly.angle = (const double*)(base + o_pa);
  d.poly.cond_off = (const uint32_t*)(base + o_po);
  d.poly.cond_cnt = (const uint32_t*)(base + o_pc);
  d.poly.conds = (const uint64_t*)(base + o_pd);
  d.uniforms = (double*)(base + o_u);
  d.status = (int32_t*)(base + o_s);
  d.outcomes = (uint8_t*)(base + o_o);

  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  if (P.n_measures) {
    if (int r = ensure(h, h->reduce, (size_t)nb * 3 * 8 + 256)) return r;
  }
  const double bpa = f64 ? 16.0 : 8.0;
  const double len = (double)(1ull << st->n);
  uint32_t mi = 0;
  const bool rec = h->record_passes;
  if (rec) {
    h->records.clear();
    const size_t need = 2 * (P.passes.size() + 1);
    while (h->events.size() < need) {
      cudaEvent_t ev;
      CK(cudaEventCreate(&ev), "event create");
      h->events.push_back(ev);
    }
  }
  auto record_begin = [&](size_t k) -> cudaError_t {
    return rec ? cudaEventRecord(h->events[2 * k], h->stream) : cudaSuccess;
  };
  auto record_end = [&](size_t k, uint32_t kind, uint32_t gates, uint32_t nq, const uint32_t* qs, uint32_t post,
                        double bytes) -> cudaError_t {
    if (!rec) return cudaSuccess;
    aleph_b200_pass_record r{};
    r.kind = kind;
    r.gates = gates;
    r.n = st->n;
    r.nq = nq;
    for (uint32_t j = 0; j < nq && j < 8; ++j) r.qubits[j] = qs[j];
    r.post_ops = post;
    r.bytes = bytes;
    h->records.push_back(r);
    return cudaEventRecord(h->events[2 * k + 1], h->stream);
  };
  size_t pk = 0;
  for (const Pass& ps : P.passes) {
    cudaError_t e = record_begin(pk);
    if (e != cudaSuccess) return cuda_fail(h, e, "event record");
    switch (ps.kind) {
      case PASS_TILE:
        e = launch_tile_pass(st->amps, st->precision, ps.tile, d.ops, d.coef, d.poly, (int*)(d.status + 4),
                             h->sm_count, h->stream);
        h->stats.tile_passes++;
        h->stats.passes++;
        h->stats.algorithmic_bytes += 2 * len * bpa;
        break;
      case PASS_SMEM:
        e = launch_smem_pass(st->amps, st->precision, st->n, d.ops + ps.tile.op_begin, ps.tile.op_count, d.coef, d.poly,
                             h->stream);
        h->stats.passes++;
        h->stats.algorithmic_bytes += 2 * len * bpa;
        break;
      case PASS_KQ:
        e = launch_kq_pass(st->amps, st->precision, st->n, d.ops + ps.tile.op_begin, P.ops[ps.tile.op_begin], d.coef,
                           h->stream);
        h->stats.passes++;
        h->stats.algorithmic_bytes += 2 * len * bpa;
        break;
      case PASS_MEASURE:
        e = launch_measure_pass(st->amps, st->precision, st->n, ps.qubit, (double*)h->reduce.ptr, nb, d.uniforms,
                                n_uniforms, d.status, d.outcomes + mi, h->stream);
        ++mi;
        h->stats.kernel_launches += 3;
        h->stats.algorithmic_bytes += 3 * len * bpa;
        break;
      case PASS_BLOCK:
        e = launch_block_pass(st->amps, ps.block, (const uint8_t*)(base + o_img), d.ops, d.coef, d.poly,
                              (int*)(d.status + 4), h->sm_count, h->stream);
        h->stats.block_passes++;
        h->stats.passes++;
        h->stats.algorithmic_bytes += 2 * len * bpa;
        break;
      case PASS_PERMUTE:
        e = launch_permute_pass(st->amps, st->precision, st->n, ps.sigma, h->sm_count, h->stream);
        h->stats.passes++;
        h->stats.algorithmic_bytes += 2 * len * bpa;
        break;
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    h->stats.kernel_launches++;
    h->stats.gates_planned += ps.gates;
    {
      const uint32_t* qs = ps.kind == PASS_BLOCK ? ps.block.bq : ps.tile.hq;
      const uint32_t nq = ps.kind == PASS_BLOCK ? 6 : ps.kind == PASS_TILE ? ps.tile.R : 0;
      const double bytes = ps.kind == PASS_MEASURE ? 3 * len * bpa : 2 * len * bpa;
      CK(record_end(pk, (uint32_t)ps.kind, ps.gates, nq, qs, ps.kind == PASS_BLOCK ? ps.block.post_count : 0, bytes),
         "event record");
      if (rec) {
        aleph_b200_pass_record& r = h->records.back();
        r.lane_ops = ps.lane_ops;
        r.dense_ops = ps.dense_ops;
        r.diag_ops = ps.diag_ops;
        r.fma_per_amp = ps.fma_per_amp;
        r.variant = ps.kind == PASS_TILE ? ps.tile.occupancy : 0;
      }
    }
    ++pk;
  }
  bool any_block = false;
  for (const Pass& ps : P.passes) any_block |= ps.kind == PASS_BLOCK;
  if (any_block && P.renormalize) {
    if (int r = ensure(h, h->reduce, (size_t)nb * 3 * 8 + 256)) return r;
    double* part = (double*)h->reduce.ptr;
    CK(record_begin(pk), "event record");
    CK(launch_renormalize(st->amps, st->precision, st->n, part, nb, part + 3 * (size_t)nb, h->stream), "renormalize");
    CK(record_end(pk, 6, 0, 0, nullptr, 0, 3 * len * bpa), "event record");
    ++pk;
    h->stats.kernel_launches += 3;
    h->stats.algorithmic_bytes += 3 * len * bpa;
  }
  if (rec) {
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
    for (size_t k = 0; k < h->records.size(); ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->events[2 * k], h->events[2 * k + 1]), "event elapsed");
      h->records[k].ms = ms;
    }
  }
  if (status_out || outcomes_out || P.n_measures || any_block) {
    std::vector<int32_t> stv(16, 0);
    CK(copy_async(h, stv.data(), d.status, 16 * 4, cudaMemcpyDeviceToHost, h->stream), "status readback");
    std::vector<uint8_t> oc(P.n_measures + 1, 0);
    if (P.n_measures)
      CK(copy_async(h, oc.data(), d.outcomes, P.n_measures, cudaMemcpyDeviceToHost, h->stream), "outcome readback");
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
    if (stv[4] != 0)  // a tile or block pass gave up on a bounded wait
      return set_error(h, ALEPH_B200_DEVICE_FAILURE, "device operation failed: pass copy wait expired");
    if (status_out) *status_out = stv;
    if (outcomes_out) {
      oc.resize(P.n_measures);
      *outcomes_out = oc;
    }
    if (stv[0] != 0 && !status_out) {
      aleph_b200_error_info e{};
      e.status = stv[0];
      e.qubit = (uint32_t)stv[2];
      return report(h, e);
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int aleph_b200_create(uint64_t seed, int device, int precision, aleph_b200_handle** out) {
  if (!out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = nullptr;
  if (precision < ALEPH_B200_F64 || precision > ALEPH_B200_TC32) return ALEPH_B200_INVALID_ARGUMENT;
  FullHandle* h = new (std::nothrow) FullHandle();
  if (!h) return ALEPH_B200_DEVICE_FAILURE;
  h->device = device;
  h->precision = precision;
  h->qubit_cap = precision == ALEPH_B200_F64 ? 33 : 34;
  h->opts.tile_r = 5;
  h->opts.tensor_blocks = precision == ALEPH_B200_TC32;
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) h->x.rng[i] = splitmix64(x);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  // Load the sampling module now, which reserves the fixed buffer of
  // aleph_b200_sample_cumulative_noalloc on this device: under lazy module
  // loading it would otherwise be reserved at that entry point's first call,
  // when the device may already be full.
  if (e == cudaSuccess) {
    void* fixed = nullptr;
    e = fixed_sample_scratch_address(&fixed);
  }
  if (e != cudaSuccess) {
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return ALEPH_B200_DEVICE_FAILURE;
  }
  *out = h;
  return ALEPH_B200_OK;
}

int aleph_b200_destroy(aleph_b200_handle* h) {
  if (!h) return ALEPH_B200_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (Scratch* s : {&h->reduce, &h->plan_buf, &h->sample, &h->status, &h->qaoa.dev, &h->qaoa.state, &h->qaoa.cuts})
    if (s->ptr) cudaFree(s->ptr);
  for (Scratch& s : h->state_pool) cudaFree(s.ptr);
  if (h->qaoa.exec) cudaGraphExecDestroy(h->qaoa.exec);
  if (h->qaoa.host_in) cudaFreeHost(h->qaoa.host_in);
  if (h->qaoa.host_out) cudaFreeHost(h->qaoa.host_out);
  for (cudaEvent_t ev : h->events) cudaEventDestroy(ev);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete static_cast<FullHandle*>(h);
  return ALEPH_B200_OK;
}

int aleph_b200_set_qubit_cap(aleph_b200_handle* h, uint32_t cap) {
  if (!h) return ALEPH_B200_INVALID_ARGUMENT;
  h->qubit_cap = cap;
  return ALEPH_B200_OK;
}

int aleph_b200_allocate(aleph_b200_handle* h, uint32_t n, aleph_b200_state** out) {
  if (!h || !out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = nullptr;
  if (n > h->qubit_cap || n > 40) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_TOO_MANY_QUBITS;
    e.requested = n;
    e.limit = h->qubit_cap;
    return report(h, e);
  }
  if (int r = bind(h)) return r;
  aleph_b200_state* st = new (std::nothrow) aleph_b200_state();
  if (!st) return set_error(h, ALEPH_B200_DEVICE_FAILURE, "host allocation failed");
  st->n = n;
  st->precision = h->precision == ALEPH_B200_F64 ? ALEPH_B200_F64 : ALEPH_B200_F32;
  st->bytes = (size_t)(st->precision == ALEPH_B200_F64 ? 16 : 8) << n;
  st->amps = nullptr;
  for (size_t k = 0; k < h->state_pool.size(); ++k)
    if (h->state_pool[k].bytes == st->bytes) {  // a freed buffer of this size: reuse it, in stream order
      st->amps = h->state_pool[k].ptr;
      h->state_pool.erase(h->state_pool.begin() + (long)k);
      break;
    }
  cudaError_t e = cudaSuccess;
  if (!st->amps) {
    e = cudaMalloc(&st->amps, st->bytes);
    if (e == cudaErrorMemoryAllocation && !h->state_pool.empty()) {  // give the pooled buffers back, retry
      cudaGetLastError();
      cudaStreamSynchronize(h->stream);
      for (Scratch& s : h->state_pool) cudaFree(s.ptr);
      h->state_pool.clear();
      e = cudaMalloc(&st->amps, st->bytes);
    }
  }
  if (e != cudaSuccess) {
    delete st;
    cudaGetLastError();
    return cuda_fail(h, e, "state allocation");
  }
  e = launch_init_zero_state(st->amps, n, st->precision, h->stream);
  if (e != cudaSuccess) {
    cudaFree(st->amps);
    delete st;
    return cuda_fail(h, e, "state init");
  }
  h->stats.kernel_launches++;
  *out = st;
  return ALEPH_B200_OK;
}

// With a handle, the buffer goes to the handle's pool (at most two are kept;
// an older one is released): later kernels on the handle's stream are
// ordered after the ones that used it, so no synchronisation is needed.
int aleph_b200_free_state(aleph_b200_handle* h, aleph_b200_state* st) {
  if (!st) return ALEPH_B200_OK;
  if (h) {
    cudaSetDevice(h->device);
    if (h->state_pool.size() >= 2) {
      cudaStreamSynchronize(h->stream);
      cudaFree(h->state_pool.front().ptr);
      h->state_pool.erase(h->state_pool.begin());
    }
    Scratch s;
    s.ptr = st->amps;
    s.bytes = st->bytes;
    h->state_pool.push_back(s);
  } else {
    cudaFree(st->amps);
  }
  delete st;
  return ALEPH_B200_OK;
}

int aleph_b200_reset_state(aleph_b200_handle* h, aleph_b200_state* st) {
  if (!h || !st) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  CK(launch_init_zero_state(st->amps, st->n, st->precision, h->stream), "state init");
  h->stats.kernel_launches++;
  return ALEPH_B200_OK;
}

int aleph_b200_num_qubits(const aleph_b200_state* st, uint32_t* out) {
  if (!st || !out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = st->n;
  return ALEPH_B200_OK;
}

int aleph_b200_apply_gate(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_instr* g, const double* pool,
                          uint64_t pool_len) {
  if (!h || !st || !g) return ALEPH_B200_INVALID_ARGUMENT;
  if (g->kind >= 28) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_UNSUPPORTED_GATE;
    std::snprintf(e.kind, sizeof(e.kind), "%s", gate_name(g->kind));
    return report(h, e);
  }
  if (int r = bind(h)) return r;
  std::vector<Lowered> ops(1);
  aleph_b200_error_info e{};
  if (lower_gate(*g, st->n, pool, pool_len, &ops[0], &e)) return report(h, e);
  const uint32_t n = st->n;
  if (g->kind == ALEPH_GATE_SWAP && g->num_controls == 0 && h->opts.relabel_swaps && n > h->opts.smem_max_n &&
      n >= 6 && n <= kMaxQubits) {
    // a SWAP of a streamed state is a permutation pass (no arithmetic; tiles
    // that the swap leaves in place are not touched)
    Lowered L;
    std::memset(&L.op, 0, sizeof(Op));
    L.is_permute = true;
    L.sigma.resize(n);
    for (uint32_t q = 0; q < n; ++q) L.sigma[q] = (uint8_t)q;
    std::swap(L.sigma[g->qubits[0]], L.sigma[g->qubits[1]]);
    L.gates = 1;
    ops[0] = std::move(L);
  }
  Plan P;
  if (int s = build_plan(ops, n, h->opts, &P)) return set_error(h, s, "optimization pipeline failed: planner");
  return execute(h, st, P, nullptr, 0, nullptr, nullptr);
}

// Appends the permutation passes that move logical qubit q from position
// phys[q] back to q (psi'(j) = psi(pi(j)), pi = phys), then resets phys.
static void settle_relabeling(std::vector<uint32_t>& phys, uint32_t& swaps, uint32_t record, std::vector<Lowered>& ops) {
  bool first = true;
  for (auto& sigma : split_into_involutions(phys)) {
    ops.emplace_back();
    Lowered& L = ops.back();
    std::memset(&L.op, 0, sizeof(Op));
    L.is_permute = true;
    L.sigma = std::move(sigma);
    L.record = record;
    L.gates = first ? swaps : 0;
    first = false;
  }
  for (uint32_t q = 0; q < (uint32_t)phys.size(); ++q) phys[q] = q;
  swaps = 0;
}

// Lowers a record stream for an n-qubit register into planner ops, validating
// every record first (crates/aleph-sv/src/backend.rs apply_gate order).
//
// With relabel_swaps, an uncontrolled SWAP moves no data: it exchanges two
// entries of the logical -> physical map `phys`, later records act on the
// mapped qubits, and the map is settled by at most two in-place permutation
// passes before a DiagonalPhase record and at the end of the stream. Errors
// still name the logical qubits of the record as written.
static int lower_stream(aleph_b200_handle* h, uint32_t n, const aleph_b200_instr* in, uint64_t count,
                        const aleph_b200_pools* pools, std::vector<Lowered>* out) {
  const double* pool = pools ? pools->matrix_pool : nullptr;
  const uint64_t pool_len = pools ? pools->matrix_pool_len : 0;
  std::vector<Lowered>& ops = *out;
  ops.reserve(count);
  // states that live in shared memory for a whole pass swap qubits for free
  const bool relabel = h->opts.relabel_swaps && n > h->opts.smem_max_n && n >= 6 && n <= kMaxQubits;
  std::vector<uint32_t> phys(n);
  for (uint32_t q = 0; q < n; ++q) phys[q] = q;
  uint32_t swaps = 0;  // SWAP records absorbed since the map was last settled
  uint64_t tiled_left = 0;  // gates of the current TiledBlock record still to come
  auto mapped = [&]() {
    for (uint32_t q = 0; q < n; ++q)
      if (phys[q] != q) return true;
    return false;
  };
  for (uint64_t i = 0; i < count; ++i) {
    const aleph_b200_instr& g = in[i];
    aleph_b200_error_info e{};
    e.instruction = (uint32_t)i;
    const bool tiled = tiled_left > 0;
    if (tiled) --tiled_left;
    if (tiled && g.kind >= 28) {
      // a TiledBlock holds gates only (crates/aleph-ir/src/tiled_block.rs)
      e.status = ALEPH_B200_INVALID_ARGUMENT;
      std::snprintf(e.kind, sizeof(e.kind), "tiled block member");
      return report(h, e);
    }
    if (g.kind < 28) {
      ops.emplace_back();
      if (lower_gate(g, n, pool, pool_len, &ops.back(), &e, tiled)) return report(h, e);
      ops.back().record = (uint32_t)i;
      if (relabel && g.kind == ALEPH_GATE_SWAP && g.num_controls == 0) {
        ops.pop_back();  // validated; the swap becomes a relabeling
        std::swap(phys[g.qubits[0]], phys[g.qubits[1]]);
        ++swaps;
        continue;
      }
      if (relabel && swaps && mapped()) {
        aleph_b200_instr gm = g;  // the same gate on the physical positions
        for (uint32_t k = 0; k < g.num_qubits && k < 8; ++k) gm.qubits[k] = phys[g.qubits[k]];
        for (uint32_t k = 0; k < g.num_controls && k < 8; ++k) gm.controls[k] = phys[g.controls[k]];
        ops.back() = Lowered{};
        if (lower_gate(gm, n, pool, pool_len, &ops.back(), &e, tiled)) return report(h, e);
        ops.back().record = (uint32_t)i;
      }
    } else if (g.kind == ALEPH_INSTR_MEASURE) {
      if (g.num_qubits != 1) {
        e.status = ALEPH_B200_INVALID_ARGUMENT;
        std::snprintf(e.kind, sizeof(e.kind), "measure record");
        return report(h, e);
      }
      if (g.qubits[0] >= n) {
        e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
        e.qubit = g.qubits[0];
        e.num_qubits = n;
        return report(h, e);
      }
      ops.emplace_back();
      std::memset(&ops.back().op, 0, sizeof(Op));
      ops.back().is_measure = true;
      ops.back().measure_qubit = relabel ? phys[g.qubits[0]] : g.qubits[0];
      ops.back().record = (uint32_t)i;
    } else if (g.kind == ALEPH_INSTR_RESET) {
      e.status = ALEPH_B200_UNSUPPORTED_INSTRUCTION;
      std::snprintf(e.kind, sizeof(e.kind), "reset");
      return report(h, e);
    } else if (g.kind == ALEPH_INSTR_BARRIER) {
      continue;  // no-op
    } else if (g.kind == ALEPH_INSTR_TILED_BLOCK) {
      // its data_len gates follow as plain records; controls at or above
      // tile_bits act as ordinary controls (the reference's executor skips
      // the tiles where they are 0, backend.rs:239-261), so the gates are
      // planned like any others
      if (g.data_len > count - i - 1) {
        e.status = ALEPH_B200_INVALID_ARGUMENT;
        std::snprintf(e.kind, sizeof(e.kind), "tiled block length");
        return report(h, e);
      }
      tiled_left = g.data_len;
      continue;
    } else if (g.kind == ALEPH_INSTR_DIAGONAL_PHASE) {
      if (!pools || g.data_offset + g.data_len > pools->n_terms || (g.data_len && !pools->terms)) {
        e.status = ALEPH_B200_INVALID_ARGUMENT;
        std::snprintf(e.kind, sizeof(e.kind), "diagonal phase terms");
        return report(h, e);
      }
      if (relabel && mapped()) settle_relabeling(phys, swaps, (uint32_t)i, ops);  // its masks are logical
      ops.emplace_back();
      if (lower_diagonal_phase(pools->terms + g.data_offset, g.data_len, pools->cond_pool, pools->n_conds, &ops.back(),
                               &e))
        return report(h, e);
      ops.back().record = (uint32_t)i;
    } else {
      e.status = ALEPH_B200_UNSUPPORTED_INSTRUCTION;
      std::snprintf(e.kind, sizeof(e.kind), "%s", gate_name(g.kind));
      return report(h, e);
    }
  }
  if (relabel && mapped()) settle_relabeling(phys, swaps, count ? (uint32_t)(count - 1) : 0, ops);
  return ALEPH_B200_OK;
}

// Runs a lowered plan with measurement variates: explicit, or drawn from the
// handle RNG (only the consumed ones advance it).
static int run_plan(aleph_b200_handle* h, aleph_b200_state* st, const Plan& P, const double* mu, uint64_t n_mu,
                    uint8_t* outcomes, uint64_t outcomes_cap, uint64_t* n_outcomes, int32_t* used_out,
                    Scratch* cache = nullptr, bool* cache_ready = nullptr) {
  std::vector<double> drawn;
  uint64_t saved[4];
  std::memcpy(saved, ext(h)->rng, sizeof(saved));
  if (!mu && P.n_measures) {
    drawn.resize(P.n_measures);
    for (auto& u : drawn) u = rng_f64(h);
    mu = drawn.data();
    n_mu = drawn.size();
  }
  std::vector<int32_t> stv;
  std::vector<uint8_t> oc;
  if (int r = execute(h, st, P, mu, (uint32_t)n_mu, &stv, &oc, cache, cache_ready)) return r;
  if (!drawn.empty()) {
    std::memcpy(ext(h)->rng, saved, sizeof(saved));
    for (int32_t k = 0; k < stv[1]; ++k) rng_next(h);
  }
  if (stv[0] != 0) {
    aleph_b200_error_info e{};
    e.status = stv[0];
    e.qubit = (uint32_t)stv[2];
    if (e.status == ALEPH_B200_INVALID_STATE)
      std::snprintf(e.kind, sizeof(e.kind), "norm drifted beyond budget");
    else if (e.status == ALEPH_B200_INVALID_ARGUMENT)
      std::snprintf(e.kind, sizeof(e.kind), "measure uniforms exhausted");
    return report(h, e);
  }
  if (outcomes)
    for (size_t i = 0; i < oc.size() && i < outcomes_cap; ++i) outcomes[i] = oc[i];
  if (n_outcomes) *n_outcomes = oc.size();
  if (used_out) *used_out = stv.empty() ? 0 : stv[1];
  return ALEPH_B200_OK;
}

static int stream_impl(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_instr* in, uint64_t count,
                       const aleph_b200_pools* pools, const double* mu, uint64_t n_mu, uint8_t* outcomes,
                       uint64_t outcomes_cap, uint64_t* n_outcomes, int32_t* used_out) {
  if (!h || !st || (!in && count)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  if (n_outcomes) *n_outcomes = 0;
  std::vector<Lowered> ops;
  if (int r = lower_stream(h, st->n, in, count, pools, &ops)) return r;
  Plan P;
  if (int s = build_plan(ops, st->n, h->opts, &P)) return set_error(h, s, "optimization pipeline failed: planner");
  return run_plan(h, st, P, mu, n_mu, outcomes, outcomes_cap, n_outcomes, used_out);
}

int aleph_b200_apply_gate_stream(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_instr* in, uint64_t count,
                                 const aleph_b200_pools* pools, const double* mu, uint64_t n_mu, uint8_t* outcomes,
                                 uint64_t outcomes_cap, uint64_t* n_outcomes) {
  return stream_impl(h, st, in, count, pools, mu, n_mu, outcomes, outcomes_cap, n_outcomes, nullptr);
}

struct aleph_b200_plan {
  uint32_t n = 0;
  Plan P;
  Scratch buf;
  bool uploaded = false;
};

int aleph_b200_compile(aleph_b200_handle* h, uint32_t num_qubits, const aleph_b200_instr* in, uint64_t count,
                       const aleph_b200_pools* pools, aleph_b200_plan** out) {
  if (!h || !out || (!in && count)) return ALEPH_B200_INVALID_ARGUMENT;
  *out = nullptr;
  if (num_qubits > h->qubit_cap || num_qubits > 40) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_TOO_MANY_QUBITS;
    e.requested = num_qubits;
    e.limit = h->qubit_cap;
    return report(h, e);
  }
  std::vector<Lowered> ops;
  if (int r = lower_stream(h, num_qubits, in, count, pools, &ops)) return r;
  aleph_b200_plan* p = new (std::nothrow) aleph_b200_plan();
  if (!p) return set_error(h, ALEPH_B200_DEVICE_FAILURE, "host allocation failed");
  p->n = num_qubits;
  if (int s = build_plan(ops, num_qubits, h->opts, &p->P)) {
    delete p;
    return set_error(h, s, "optimization pipeline failed: planner");
  }
  *out = p;
  return ALEPH_B200_OK;
}

int aleph_b200_execute(aleph_b200_handle* h, aleph_b200_state* st, aleph_b200_plan* plan, const double* mu,
                       uint64_t n_mu, uint8_t* outcomes, uint64_t outcomes_cap, uint64_t* n_outcomes) {
  if (!h || !st || !plan) return ALEPH_B200_INVALID_ARGUMENT;
  if (n_outcomes) *n_outcomes = 0;
  if (plan->n != st->n)
    return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "plan compiled for %u qubits, state has %u", plan->n, st->n);
  if (int r = bind(h)) return r;
  return run_plan(h, st, plan->P, mu, n_mu, outcomes, outcomes_cap, n_outcomes, nullptr, &plan->buf, &plan->uploaded);
}

int aleph_b200_plan_free(aleph_b200_handle* h, aleph_b200_plan* plan) {
  if (!plan) return ALEPH_B200_OK;
  if (plan->buf.ptr) {
    if (h) {
      cudaSetDevice(h->device);
      cudaStreamSynchronize(h->stream);
    }
    cudaFree(plan->buf.ptr);
  }
  delete plan;
  return ALEPH_B200_OK;
}

// ---- out-of-core runs --------------------------------------------------------
// crates/aleph-cuda/src/sv/paged.rs:1-38 (tiling scheme), :138-251
// (run_paged), :253-276 (run_paged_overlapped). The reference gathers the
// tiles of one gate at a time; here a segment of gates shares one gather, so
// the host state is read and written once per segment, not once per gate.
struct aleph_b200_paged_state {
  uint32_t n = 0;
  int precision = ALEPH_B200_F64;
  void* host = nullptr;  // pinned, 2^n amplitudes
  size_t bytes = 0;
  aleph_b200_paged_info info{};
};

namespace {

uint64_t deposit_bits(uint64_t v, const std::vector<uint32_t>& positions) {  // bit i of v -> bit positions[i]
  uint64_t r = 0;
  for (size_t i = 0; i < positions.size(); ++i) r |= ((v >> i) & 1) << positions[i];
  return r;
}

uint64_t qubit_mask(const aleph_b200_instr& r, uint32_t n) {  // targets and controls
  uint64_t mask = 0;
  for (uint32_t k = 0; k < r.num_qubits && k < 8; ++k)
    if (r.qubits[k] < n) mask |= 1ull << r.qubits[k];
  for (uint32_t k = 0; k < r.num_controls && k < 8; ++k)
    if (r.controls[k] < n) mask |= 1ull << r.controls[k];
  return mask;
}
uint64_t high_mask(const aleph_b200_instr& r, uint32_t m, uint32_t n) {
  return qubit_mask(r, n) & ~((1ull << m) - 1);
}

// Segments of an out-of-core run: each takes, in order, every remaining gate
// whose high qubits (>= m) fit the budget together with the segment's, and
// that shares no qubit with a gate the segment leaves for later, so it
// commutes with all of them and the reordering is exact. Barriers are dropped.
struct PagedSegment {
  std::vector<uint64_t> gates;  // instruction indices, in execution order
  uint64_t hmask = 0;           // the high qubits the segment gathers
};
std::vector<PagedSegment> paged_segments(const aleph_b200_instr* in, uint64_t count, uint32_t n, uint32_t m,
                                         uint32_t g_budget) {
  std::vector<PagedSegment> segs;
  std::vector<uint64_t> remaining, deferred;
  for (uint64_t i = 0; i < count; ++i)
    if (in[i].kind != ALEPH_INSTR_BARRIER) remaining.push_back(i);
  while (!remaining.empty()) {
    PagedSegment sg;
    uint64_t blocked = 0;
    deferred.clear();
    for (uint64_t i : remaining) {
      const uint64_t qm = qubit_mask(in[i], n), gm = qm & ~((1ull << m) - 1);
      if (!(qm & blocked) && (uint32_t)__builtin_popcountll(sg.hmask | gm) <= g_budget) {
        sg.gates.push_back(i);
        sg.hmask |= gm;
      } else {
        deferred.push_back(i);
        blocked |= qm;
      }
    }
    segs.push_back(std::move(sg));
    remaining.swap(deferred);
  }
  return segs;
}

struct PagedRing {
  int device = 0;
  std::vector<void*> buf;
  std::vector<cudaEvent_t> in, done, out;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  ~PagedRing() {
    cudaSetDevice(device);
    if (h2d) cudaStreamSynchronize(h2d);
    if (d2h) cudaStreamSynchronize(d2h);
    for (void* p : buf) cudaFree(p);
    for (auto* v : {&in, &done, &out})
      for (cudaEvent_t e : *v) cudaEventDestroy(e);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }
};

}  // namespace

int aleph_b200_paged_run(aleph_b200_handle* h, uint32_t n, const aleph_b200_instr* in, uint64_t count,
                         const aleph_b200_pools* pools, uint32_t m, uint32_t depth, aleph_b200_paged_state** out) {
  if (!h || !out || (!in && count)) return ALEPH_B200_INVALID_ARGUMENT;
  *out = nullptr;
  if (n == 0 && count == 0) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_EMPTY_CIRCUIT;
    return report(h, e);
  }
  if (m == 0 || m >= n) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_STATE;
    std::snprintf(e.kind, sizeof(e.kind), "paged: need 1<=tile_qubits<n");
    return report(h, e);
  }
  if (n > kMaxQubits) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_TOO_MANY_QUBITS;
    e.requested = n;
    e.limit = kMaxQubits;
    return report(h, e);
  }
  if (depth == 0) depth = 3;
  if (depth > 8) depth = 8;
  // one scan (paged.rs:161-185): unsupported instructions, the widest gate
  uint32_t g_max = 0;
  for (uint64_t i = 0; i < count; ++i) {
    const char* kind = nullptr;
    switch (in[i].kind) {
      case ALEPH_INSTR_MEASURE: kind = "measure"; break;
      case ALEPH_INSTR_RESET: kind = "reset"; break;
      case ALEPH_INSTR_DIAGONAL_PHASE: kind = "diagonal-phase"; break;
      case ALEPH_INSTR_TILED_BLOCK: kind = "tiled-block"; break;
      case ALEPH_INSTR_BARRIER: continue;
      default: break;
    }
    if (kind) {
      aleph_b200_error_info e{};
      e.status = ALEPH_B200_UNSUPPORTED_INSTRUCTION;
      e.instruction = i;
      std::snprintf(e.kind, sizeof(e.kind), "%s", kind);
      return report(h, e);
    }
    g_max = std::max<uint32_t>(g_max, (uint32_t)__builtin_popcountll(high_mask(in[i], m, n)));
  }
  if (int r = bind(h)) return r;
  const int prec = h->precision == ALEPH_B200_F64 ? ALEPH_B200_F64 : ALEPH_B200_F32;
  const size_t bpa = prec == ALEPH_B200_F64 ? 16 : 8;
  // the largest tile group the device holds: `depth` buffers in half of the free memory
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b), "memory info");
  uint32_t L = std::min<uint32_t>(n, std::min<uint32_t>(h->qubit_cap, kMaxQubits));
  if (h->paged_local_max) L = std::min<uint32_t>(L, std::max<uint32_t>(h->paged_local_max, m));
  while (L > m && (double)depth * (double)(bpa << L) > 0.5 * (double)free_b) --L;
  if (m + g_max > L || (double)depth * (double)(bpa << m) > 0.5 * (double)free_b) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_TOO_MANY_QUBITS;
    e.requested = m + g_max;
    e.limit = L;
    return report(h, e);
  }
  const uint32_t g_budget = L - m;
  // every gate validated against the full register first (same checks and
  // payloads as the in-core stream); nothing is allocated before this passes
  {
    std::vector<Lowered> ops;
    if (int r = lower_stream(h, n, in, count, pools, &ops)) return r;
  }
  const std::vector<PagedSegment> segs = paged_segments(in, count, n, m, g_budget);
  uint32_t l_used = m;
  for (const PagedSegment& sg : segs) l_used = std::max<uint32_t>(l_used, m + (uint32_t)__builtin_popcountll(sg.hmask));

  aleph_b200_paged_state* ps = new (std::nothrow) aleph_b200_paged_state();
  if (!ps) return set_error(h, ALEPH_B200_DEVICE_FAILURE, "host allocation failed");
  ps->n = n;
  ps->precision = prec;
  ps->bytes = bpa << n;
  cudaError_t ce = cudaHostAlloc(&ps->host, ps->bytes, cudaHostAllocPortable);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    delete ps;
    return cuda_fail(h, ce, "pinned host state allocation");
  }
  // The first segment generates |0...0> on the device and its scatters write
  // every tile, so the host state is only initialised when no gate runs.
  if (segs.empty()) {
    std::memset(ps->host, 0, ps->bytes);
    if (prec == ALEPH_B200_F64) ((double*)ps->host)[0] = 1.0;
    else ((float*)ps->host)[0] = 1.0f;
  }
  static const double kOne64[2] = {1.0, 0.0};
  static const float kOne32[2] = {1.0f, 0.0f};
  PagedRing ring;
  ring.device = h->device;
  Scratch plan_buf;  // the current segment's uploaded plan tables
  // on failure: no copy into or out of the host state may still be in
  // flight when it is freed
  auto fail = [&](int r) {
    if (ring.h2d) cudaStreamSynchronize(ring.h2d);
    if (ring.d2h) cudaStreamSynchronize(ring.d2h);
    cudaStreamSynchronize(h->stream);
    if (plan_buf.ptr) cudaFree(plan_buf.ptr);
    plan_buf = Scratch{};
    aleph_b200_paged_free(ps);
    return r;
  };
  const auto t0 = std::chrono::steady_clock::now();

  const size_t buf_bytes = bpa << l_used;
  ring.buf.assign(depth, nullptr);
  ring.in.assign(depth, nullptr);
  ring.done.assign(depth, nullptr);
  ring.out.assign(depth, nullptr);
  for (uint32_t k = 0; k < depth; ++k) {
    if ((ce = cudaMalloc(&ring.buf[k], buf_bytes)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&ring.in[k], cudaEventDisableTiming)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&ring.done[k], cudaEventDisableTiming)) != cudaSuccess ||
        (ce = cudaEventCreateWithFlags(&ring.out[k], cudaEventDisableTiming)) != cudaSuccess) {
      cudaGetLastError();
      return fail(cuda_fail(h, ce, "paged device ring"));
    }
  }
  if ((ce = cudaStreamCreateWithFlags(&ring.h2d, cudaStreamNonBlocking)) != cudaSuccess ||
      (ce = cudaStreamCreateWithFlags(&ring.d2h, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(cuda_fail(h, ce, "paged copy streams"));

  const size_t tile_bytes = bpa << m;
  uint64_t group = 0;  // global group counter: ring slot = group % depth
  aleph_b200_paged_info& info = ps->info;
  info.num_qubits = n;
  info.tile_qubits = m;
  info.local_qubits = l_used;
  info.depth = depth;
  std::vector<aleph_b200_instr> local;
  for (size_t si = 0; si < segs.size(); ++si) {
    const PagedSegment& sg = segs[si];
    std::vector<uint32_t> H, R;  // the segment's high qubits / the other high qubits, ascending
    for (uint32_t q = m; q < n; ++q) ((sg.hmask >> q) & 1 ? H : R).push_back(q);
    const uint32_t hh = (uint32_t)H.size(), nl = m + hh;
    std::vector<uint32_t> to_local(n);
    for (uint32_t q = 0; q < m; ++q) to_local[q] = q;
    for (uint32_t r = 0; r < hh; ++r) to_local[H[r]] = m + r;
    // the segment on its local register, compiled once
    local.clear();
    for (uint64_t i : sg.gates) local.push_back(in[i]);
    for (aleph_b200_instr& r : local) {
      for (uint32_t k = 0; k < r.num_qubits && k < 8; ++k) r.qubits[k] = to_local[r.qubits[k]];
      for (uint32_t k = 0; k < r.num_controls && k < 8; ++k) r.controls[k] = to_local[r.controls[k]];
    }
    Plan P;
    {
      std::vector<Lowered> ops;
      if (int r = lower_stream(h, nl, local.data(), local.size(), pools, &ops)) return fail(r);
      if (int s = build_plan(ops, nl, h->opts, &P)) return fail(set_error(h, s, "optimization pipeline failed: planner"));
      P.renormalize = false;
    }
    bool uploaded = false;
    // tile index bit (q - m) <-> qubit q
    std::vector<uint32_t> hbit(hh), rbit(R.size());
    for (uint32_t r = 0; r < hh; ++r) hbit[r] = H[r] - m;
    for (size_t r = 0; r < R.size(); ++r) rbit[r] = R[r] - m;
    const uint64_t n_outer = 1ull << R.size(), n_sub = 1ull << hh;
    auto copies = [&](uint64_t outer, uint32_t slot, bool to_device) -> cudaError_t {
      const uint64_t base = deposit_bits(outer, rbit);
      for (uint64_t s = 0; s < n_sub; ++s) {
        const uint64_t tile = base | deposit_bits(s, hbit);
        char* hp = (char*)ps->host + tile * tile_bytes;
        char* dp = (char*)ring.buf[slot] + s * tile_bytes;
        const cudaError_t e = to_device
                                  ? cudaMemcpyAsync(dp, hp, tile_bytes, cudaMemcpyHostToDevice, ring.h2d)
                                  : cudaMemcpyAsync(hp, dp, tile_bytes, cudaMemcpyDeviceToHost, ring.d2h);
        if (e != cudaSuccess) return e;
      }
      (to_device ? info.h2d_bytes : info.d2h_bytes) += n_sub * tile_bytes;
      return cudaSuccess;
    };
    // gather of group g (outer index o): waits for the slot's previous scatter
    // and, for a segment's first group, for every scatter of the segment
    // before (the tiles it reads were written there; d2h is in order)
    // (the first segment generates its groups: zeros, and amplitude 1 at
    // index 0, which sits at offset 0 of outer group 0)
    const bool generate = si == 0;
    auto gather = [&](uint64_t g, uint64_t o, bool first_of_segment) -> cudaError_t {
      const uint32_t slot = (uint32_t)(g % depth);
      cudaError_t e = cudaSuccess;
      if (g >= depth) e = cudaStreamWaitEvent(ring.h2d, ring.out[slot], 0);
      if (e == cudaSuccess && first_of_segment && g > 0)
        e = cudaStreamWaitEvent(ring.h2d, ring.out[(g - 1) % depth], 0);
      if (e == cudaSuccess && generate) {
        e = cudaMemsetAsync(ring.buf[slot], 0, n_sub * tile_bytes, ring.h2d);
        if (e == cudaSuccess && o == 0)
          e = cudaMemcpyAsync(ring.buf[slot], prec == ALEPH_B200_F64 ? (const void*)kOne64 : (const void*)kOne32, bpa,
                              cudaMemcpyHostToDevice, ring.h2d);
      } else if (e == cudaSuccess) {
        e = copies(o, slot, true);
      }
      if (e == cudaSuccess) e = cudaEventRecord(ring.in[slot], ring.h2d);
      return e;
    };
    const uint64_t g0 = group;
    CK_OR(gather(g0, 0, true), fail, "paged gather");
    for (uint64_t o = 0; o < n_outer; ++o) {
      const uint64_t g = g0 + o;
      const uint32_t slot = (uint32_t)(g % depth);
      // the next group's gather runs while this one computes (another slot)
      if (depth > 1 && o + 1 < n_outer) CK_OR(gather(g + 1, o + 1, false), fail, "paged gather");
      CK_OR(cudaStreamWaitEvent(h->stream, ring.in[slot], 0), fail, "stream wait");
      aleph_b200_state st;
      st.n = nl;
      st.precision = prec;
      st.amps = ring.buf[slot];
      st.bytes = bpa << nl;
      if (int r = run_plan(h, &st, P, nullptr, 0, nullptr, 0, nullptr, nullptr, &plan_buf, &uploaded)) return fail(r);
      CK_OR(cudaEventRecord(ring.done[slot], h->stream), fail, "event record");
      CK_OR(cudaStreamWaitEvent(ring.d2h, ring.done[slot], 0), fail, "stream wait");
      CK_OR(copies(o, slot, false), fail, "paged scatter");
      CK_OR(cudaEventRecord(ring.out[slot], ring.d2h), fail, "event record");
      if (depth == 1 && o + 1 < n_outer) CK_OR(gather(g + 1, o + 1, false), fail, "paged gather");
    }
    group += n_outer;
    info.groups += n_outer;
    ++info.segments;
    cudaStreamSynchronize(h->stream);
    if (plan_buf.ptr) cudaFree(plan_buf.ptr);
    plan_buf = Scratch{};
  }
  CK_OR(cudaStreamSynchronize(ring.d2h), fail, "stream synchronize");
  CK_OR(cudaStreamSynchronize(ring.h2d), fail, "stream synchronize");
  info.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  *out = ps;
  return ALEPH_B200_OK;
}

int aleph_b200_paged_info_get(const aleph_b200_paged_state* ps, aleph_b200_paged_info* out) {
  if (!ps || !out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = ps->info;
  return ALEPH_B200_OK;
}

int aleph_b200_paged_get_amplitudes(const aleph_b200_paged_state* ps, double* out) {
  if (!ps || !out) return ALEPH_B200_INVALID_ARGUMENT;
  const uint64_t len = 1ull << ps->n;
  if (ps->precision == ALEPH_B200_F64) {
    std::memcpy(out, ps->host, ps->bytes);
  } else {
    const float* f = (const float*)ps->host;
    for (uint64_t i = 0; i < 2 * len; ++i) out[i] = f[i];
  }
  return ALEPH_B200_OK;
}

int aleph_b200_paged_norm_sqr(const aleph_b200_paged_state* ps, double* out) {
  if (!ps || !out) return ALEPH_B200_INVALID_ARGUMENT;
  // blocks of 4096 squares summed plainly, block sums added with Kahan
  // compensation: the rounding error stays near that of one block, not of
  // a 2^(n+1)-term running sum
  const uint64_t count = 2ull << ps->n;
  double total = 0.0, comp = 0.0;
  for (uint64_t b = 0; b < count; b += 4096) {
    const uint64_t e = std::min<uint64_t>(count, b + 4096);
    double blk = 0.0;
    if (ps->precision == ALEPH_B200_F64) {
      const double* d = (const double*)ps->host;
      for (uint64_t i = b; i < e; ++i) blk += d[i] * d[i];
    } else {
      const float* f = (const float*)ps->host;
      for (uint64_t i = b; i < e; ++i) blk += (double)f[i] * (double)f[i];
    }
    const double y = blk - comp, t = total + y;
    comp = (t - total) - y;
    total = t;
  }
  *out = total;
  return ALEPH_B200_OK;
}

int aleph_b200_paged_free(aleph_b200_paged_state* ps) {
  if (!ps) return ALEPH_B200_OK;
  if (ps->host) cudaFreeHost(ps->host);
  delete ps;
  return ALEPH_B200_OK;
}

int aleph_b200_describe_paged(uint32_t n, const aleph_b200_instr* in, uint64_t count, uint32_t tile_qubits,
                              uint32_t local_qubits, uint64_t* segment_of, uint64_t* position_of,
                              uint64_t* n_segments) {
  if ((!in && count) || !n_segments || tile_qubits == 0 || tile_qubits >= n || n > kMaxQubits ||
      local_qubits < tile_qubits)
    return ALEPH_B200_INVALID_ARGUMENT;
  uint32_t g_max = 0;
  for (uint64_t i = 0; i < count; ++i)
    if (in[i].kind != ALEPH_INSTR_BARRIER)
      g_max = std::max<uint32_t>(g_max, (uint32_t)__builtin_popcountll(high_mask(in[i], tile_qubits, n)));
  if (tile_qubits + g_max > local_qubits) return ALEPH_B200_TOO_MANY_QUBITS;
  const std::vector<PagedSegment> segs = paged_segments(in, count, n, tile_qubits, local_qubits - tile_qubits);
  for (uint64_t i = 0; i < count; ++i) {
    if (segment_of) segment_of[i] = UINT64_MAX;
    if (position_of) position_of[i] = UINT64_MAX;
  }
  uint64_t pos = 0;
  for (size_t si = 0; si < segs.size(); ++si)
    for (uint64_t i : segs[si].gates) {
      if (segment_of) segment_of[i] = si;
      if (position_of) position_of[i] = pos;
      ++pos;
    }
  *n_segments = segs.size();
  return ALEPH_B200_OK;
}

int aleph_b200_qaoa_sweep(aleph_b200_handle* h, uint32_t p, const aleph_b200_qaoa_set* sets, uint32_t n_sets,
                          const uint32_t* edges, uint64_t n_edge_pairs, const double* angles, double* expectations) {
  if (!h || (n_sets && (!sets || !angles || !expectations)) || (n_edge_pairs && !edges)) return ALEPH_B200_INVALID_ARGUMENT;
  if (p == 0) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "qaoa sweep needs p >= 1 layers");
  if (n_sets == 0) return ALEPH_B200_OK;
  // validation, in the reference's order for one circuit: qubit count, then
  // each edge's CNOT(i, j) operands, then the Rz / Rx angles
  const int prec = h->precision == ALEPH_B200_F64 ? ALEPH_B200_F64 : ALEPH_B200_F32;
  const uint32_t smem_n = qaoa_smem_max_n(prec);
  uint32_t nmax_stream = 0;
  for (uint32_t k = 0; k < n_sets; ++k) {
    const aleph_b200_qaoa_set& s = sets[k];
    aleph_b200_error_info e{};
    e.instruction = k;
    if (s.num_qubits == 0 || s.num_qubits > 26) {
      e.status = ALEPH_B200_TOO_MANY_QUBITS;
      e.requested = s.num_qubits;
      e.limit = 26;
      if (s.num_qubits == 0) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "qaoa set %u has no qubits", k);
      return report(h, e);
    }
    if (s.num_edges > 128 || s.edge_offset + s.num_edges > n_edge_pairs)
      return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "qaoa set %u: edge range outside the edge pool (or > 128)", k);
    for (uint32_t j = 0; j < s.num_edges; ++j) {
      const uint32_t u = edges[2 * (s.edge_offset + j)], v = edges[2 * (s.edge_offset + j) + 1];
      if (u >= s.num_qubits || v >= s.num_qubits) {
        e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
        e.qubit = u >= s.num_qubits ? u : v;
        e.num_qubits = s.num_qubits;
        return report(h, e);
      }
      if (u == v) {
        e.status = ALEPH_B200_DUPLICATE_QUBIT;
        e.qubit = u;
        return report(h, e);
      }
    }
    for (uint32_t j = 0; j < 2 * p; ++j)
      if (!std::isfinite(angles[(size_t)2 * p * k + j])) {
        e.status = ALEPH_B200_NON_FINITE_PARAM;
        std::snprintf(e.kind, sizeof(e.kind), j < p ? "rz" : "rx");
        return report(h, e);
      }
    if (s.num_qubits > smem_n && s.num_qubits > nmax_stream) nmax_stream = s.num_qubits;
  }
  if (int r = bind(h)) return r;
  auto& Q = h->qaoa;
  // streamed sets: one state slice and one cut slice per CTA, within a memory budget
  const uint64_t slice = nmax_stream ? (1ull << nmax_stream) : 0;
  const size_t bpa = prec == ALEPH_B200_F64 ? 16 : 8;
  int grid = h->sm_count * qaoa_ctas_per_sm(prec);
  if (slice) {
    const uint64_t budget = 48ull << 30;
    const uint64_t per_cta = slice * (bpa + 1);
    if ((uint64_t)grid * per_cta > budget) grid = (int)(budget / per_cta);
    if (grid < 1) grid = 1;
  }
  // device input region: sets | order | edges | angles | out | counter
  const size_t b_sets = al((size_t)n_sets * sizeof(aleph_b200_qaoa_set)), b_order = al((size_t)n_sets * 4),
               b_edges = al((size_t)n_edge_pairs * 8), b_ang = al((size_t)n_sets * 2 * p * 8),
               b_out = al((size_t)n_sets * 8), b_cnt = al(4);
  const size_t in_bytes = b_sets + b_order + b_edges + b_ang;
  const size_t total = in_bytes + b_out + b_cnt;
  const uint64_t key[6] = {(uint64_t)prec, n_sets, p, n_edge_pairs, (uint64_t)grid, slice};
  const bool same = Q.exec && std::memcmp(key, Q.key, sizeof(key)) == 0;
  if (!same) {
    if (Q.exec) {
      cudaGraphExecDestroy(Q.exec);
      Q.exec = nullptr;
    }
    if (int r = ensure(h, Q.dev, total)) return r;
    if (slice) {
      if (int r = ensure(h, Q.state, (size_t)grid * slice * bpa)) return r;
      if (int r = ensure(h, Q.cuts, (size_t)grid * slice)) return r;
    }
    if (Q.host_in_bytes < in_bytes) {
      if (Q.host_in) cudaFreeHost(Q.host_in);
      Q.host_in = nullptr;
      Q.host_in_bytes = 0;
      CK(cudaHostAlloc(&Q.host_in, in_bytes, cudaHostAllocDefault), "pinned staging");
      Q.host_in_bytes = in_bytes;
    }
    if (Q.host_out_bytes < b_out) {
      if (Q.host_out) cudaFreeHost(Q.host_out);
      Q.host_out = nullptr;
      Q.host_out_bytes = 0;
      CK(cudaHostAlloc(&Q.host_out, b_out, cudaHostAllocDefault), "pinned staging");
      Q.host_out_bytes = b_out;
    }
  }
  // stage this call's inputs (the graph copies the staging area as it is at replay)
  uint8_t* hin = (uint8_t*)Q.host_in;
  std::memcpy(hin, sets, (size_t)n_sets * sizeof(aleph_b200_qaoa_set));
  {
    std::vector<uint32_t> order(n_sets);
    for (uint32_t k = 0; k < n_sets; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return sets[x].num_qubits > sets[y].num_qubits; });
    std::memcpy(hin + b_sets, order.data(), (size_t)n_sets * 4);
  }
  if (n_edge_pairs) std::memcpy(hin + b_sets + b_order, edges, (size_t)n_edge_pairs * 8);
  std::memcpy(hin + b_sets + b_order + b_edges, angles, (size_t)n_sets * 2 * p * 8);
  char* d = (char*)Q.dev.ptr;
  if (!same) {
    // capture: inputs up, counter cleared, the persistent sweep, results down
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t e = cudaMemcpyAsync(d, hin, in_bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + in_bytes + b_out, 0, 4, h->stream);
    if (e == cudaSuccess)
      e = launch_qaoa_sweep(prec, (const aleph_b200_qaoa_set*)d, (const uint32_t*)(d + b_sets + b_order),
                            (const double*)(d + b_sets + b_order + b_edges), (const uint32_t*)(d + b_sets),
                            (uint32_t*)(d + in_bytes + b_out), (double*)(d + in_bytes), Q.state.ptr,
                            (uint8_t*)Q.cuts.ptr, slice, n_sets, p, grid, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(Q.host_out, d + in_bytes, (size_t)n_sets * 8, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&Q.exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      Q.exec = nullptr;
      cudaGetLastError();
      return cuda_fail(h, e, "qaoa sweep graph");
    }
    std::memcpy(Q.key, key, sizeof(key));
  }
  CK(cudaGraphLaunch(Q.exec, h->stream), "qaoa sweep graph launch");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  std::memcpy(expectations, Q.host_out, (size_t)n_sets * 8);
  h->stats.kernel_launches += 1;
  h->stats.h2d_bytes += in_bytes;
  h->stats.d2h_bytes += (size_t)n_sets * 8;
  return ALEPH_B200_OK;
}

int aleph_b200_apply_diagonal_phase(aleph_b200_handle* h, aleph_b200_state* st, const aleph_b200_phase_term* terms,
                                    uint64_t n_terms, const uint64_t* conds, uint64_t n_conds) {
  if (!h || !st || (!terms && n_terms)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  std::vector<Lowered> ops(1);
  aleph_b200_error_info e{};
  if (lower_diagonal_phase(terms, n_terms, conds, n_conds, &ops[0], &e)) return report(h, e);
  Plan P;
  if (int s = build_plan(ops, st->n, h->opts, &P)) return set_error(h, s, "optimization pipeline failed: planner");
  return execute(h, st, P, nullptr, 0, nullptr, nullptr);
}

// In place, as at most two involution passes (no second state buffer).
int aleph_b200_unpermute(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* perm, uint32_t n) {
  if (!h || !st || !perm) return ALEPH_B200_INVALID_ARGUMENT;
  if (n != st->n) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "perm length %u != num_qubits %u", n, st->n);
  uint64_t seen = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (perm[i] >= n || ((seen >> perm[i]) & 1))
      return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "perm is not a permutation of 0..%u", n);
    seen |= 1ull << perm[i];
  }
  if (int r = bind(h)) return r;
  Plan P;
  for (auto& sigma : split_into_involutions(std::vector<uint32_t>(perm, perm + n))) {
    Pass ps{};
    ps.kind = PASS_PERMUTE;
    for (uint32_t q = 0; q < n; ++q) ps.sigma[q] = sigma[q];
    P.passes.push_back(ps);
  }
  if (P.passes.empty()) return ALEPH_B200_OK;
  return execute(h, st, P, nullptr, 0, nullptr, nullptr);
}

int aleph_b200_measure(aleph_b200_handle* h, aleph_b200_state* st, uint32_t qubit, double u, int* outcome,
                       int* consumed) {
  if (!h || !st || !outcome) return ALEPH_B200_INVALID_ARGUMENT;
  if (qubit >= st->n) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
    e.qubit = qubit;
    e.num_qubits = st->n;
    return report(h, e);
  }
  aleph_b200_instr rec{};
  rec.kind = ALEPH_INSTR_MEASURE;
  rec.num_qubits = 1;
  rec.qubits[0] = qubit;
  uint8_t oc = 0;
  uint64_t nout = 0;
  int32_t used = 0;
  const int r = u < 0.0 ? stream_impl(h, st, &rec, 1, nullptr, nullptr, 0, &oc, 1, &nout, &used)
                        : stream_impl(h, st, &rec, 1, nullptr, &u, 1, &oc, 1, &nout, &used);
  if (r) return r;
  *outcome = oc;
  if (consumed) *consumed = used;
  return ALEPH_B200_OK;
}

static int check_norm_host(aleph_b200_handle* h, aleph_b200_state* st, double* norm_out) {
  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  if (int r = ensure(h, h->reduce, (size_t)nb * 3 * 8 + 256)) return r;
  double* part = (double*)h->reduce.ptr;
  double* out2 = part + 3 * (size_t)nb;
  CK(launch_norm(st->amps, st->precision, st->n, part, nb, out2, h->stream), "norm");
  h->stats.kernel_launches += 2;
  double res[2];
  CK(copy_async(h, res, out2, 16, cudaMemcpyDeviceToHost, h->stream), "norm readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  if (norm_out) *norm_out = res[0];
  if (res[1] > 0.0) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_STATE;
    std::snprintf(e.kind, sizeof(e.kind), "non-finite amplitude norm2");
    return report(h, e);
  }
  if (!std::isfinite(res[0]) || std::fabs(res[0] - 1.0) > norm_tolerance(1ull << st->n, st->precision)) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_STATE;
    std::snprintf(e.kind, sizeof(e.kind), "state norm2 deviates from 1");
    return report(h, e);
  }
  return 0;
}

// status[2] of a CUMULATIVE sampling call: its shots inside the guard band
static void count_guard_band(aleph_b200_handle* h, uint32_t n, const int32_t* status) {
  h->stats.guard_band_shots += (uint32_t)status[2];
  if (n > kExactCumulativeMaxN) h->stats.guard_band_inexact += (uint32_t)status[2];
}

int aleph_b200_sample(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots, int mode, const void* variates,
                      uint64_t* out) {
  if (!h || !st || (shots && (!variates || !out))) return ALEPH_B200_INVALID_ARGUMENT;
  if (mode == ALEPH_B200_SAMPLE_AUTO) mode = shots >= 2 ? ALEPH_B200_SAMPLE_ALIAS : ALEPH_B200_SAMPLE_CUMULATIVE;
  if (mode != ALEPH_B200_SAMPLE_ALIAS && mode != ALEPH_B200_SAMPLE_CUMULATIVE)
    return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "unknown sample mode %d", mode);
  if (mode == ALEPH_B200_SAMPLE_ALIAS && st->n > 28)
    return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "alias sampling supports n <= 28; use CUMULATIVE");
  if (int r = bind(h)) return r;
  if (shots == 0) return check_norm_host(h, st, nullptr);
  const size_t sb = sample_scratch_bytes(st->n, mode, shots);
  const size_t vb = (size_t)shots * 8;
  if (int r = ensure(h, h->sample, al(sb) + 2 * al(vb) + 256)) return r;
  char* base = (char*)h->sample.ptr;
  void* dvar = base + al(sb);
  uint64_t* dout = (uint64_t*)(base + al(sb) + al(vb));
  int32_t* dstatus = (int32_t*)(base + al(sb) + 2 * al(vb));
  CK(cudaMemsetAsync(dstatus, 0, 64, h->stream), "status clear");
  CK(cudaMemsetAsync(base, 0, sb, h->stream), "scratch clear");
  CK(copy_async(h, dvar, variates, vb, cudaMemcpyHostToDevice, h->stream), "variates upload");
  CK(launch_sample(st->amps, st->precision, st->n, shots, mode, dvar, dout, base, sb, dstatus, h->sm_count, h->stream),
     "sample");
  h->stats.kernel_launches += mode == ALEPH_B200_SAMPLE_ALIAS ? 7 : 5;
  int32_t status[4];
  CK(copy_async(h, status, dstatus, 16, cudaMemcpyDeviceToHost, h->stream), "status readback");
  CK(copy_async(h, out, dout, vb, cudaMemcpyDeviceToHost, h->stream), "sample readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  if (mode == ALEPH_B200_SAMPLE_CUMULATIVE) count_guard_band(h, st->n, status);
  if (status[0]) {
    aleph_b200_error_info e{};
    e.status = status[0];
    std::snprintf(e.kind, sizeof(e.kind), "state norm2 deviates from 1");
    return report(h, e);
  }
  return ALEPH_B200_OK;
}

// Seeded sampling draws from the handle's own generator, so it is free to pick
// the faster exact method: an alias table (one u64 per shot) while the
// table's sequential construction is cheap (n <= 20, tens of ms), otherwise
// the parallel inverse CDF (one f64 per shot), which also serves every n
// above the alias limit of 28.
constexpr uint32_t kSeededAliasMaxN = 20;

int aleph_b200_sample_seeded(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots, uint64_t* out) {
  if (!h || !st || (shots && !out)) return ALEPH_B200_INVALID_ARGUMENT;
  if (shots >= 2 && st->n <= kSeededAliasMaxN) {
    std::vector<uint64_t> w(shots);
    for (auto& x : w) x = rng_next(h);
    return aleph_b200_sample(h, st, shots, ALEPH_B200_SAMPLE_ALIAS, w.data(), out);
  }
  std::vector<double> u(shots ? shots : 1, 0.0);
  for (uint32_t k = 0; k < shots; ++k) u[k] = rng_f64(h);
  return aleph_b200_sample(h, st, shots, ALEPH_B200_SAMPLE_CUMULATIVE, u.data(), out);
}

// ---- cumulative sampling from a fixed device buffer (no allocation) ------------
// The same kernels as aleph_b200_sample(CUMULATIVE), but every device byte it
// uses lives in one file-scope __device__ array reserved at module load
// (kFixedSampleScratchBytes), never in the handle's grow-on-demand scratch.
// It serves callers that cannot allocate at that point: a caller whose state
// vectors already fill HBM (a cudaMalloc after the circuit ran would fail for
// lack of memory), and a caller sampling resident states in a latency-bound
// loop, where the allocating path's scratch growth (cudaFree + cudaMalloc)
// would synchronise the whole device and stall other streams.
namespace {
// Address of the current device's fixed buffer (bind() made the handle's
// device current). Looked up on every call: the lookup is cheap once the
// module is loaded (aleph_b200_create loads it), and a cached address would
// go stale if the host program reset the device.
int fixed_base(aleph_b200_handle* h, char** out) {
  void* p = nullptr;
  cudaError_t e = fixed_sample_scratch_address(&p);
  if (e != cudaSuccess || !p) return cuda_fail(h, e != cudaSuccess ? e : cudaErrorInvalidSymbol, "fixed buffer address");
  *out = (char*)p;
  return ALEPH_B200_OK;
}
}  // namespace

int aleph_b200_sample_cumulative_noalloc(aleph_b200_handle* h, aleph_b200_state* st, uint32_t shots,
                                         const double* variates, uint64_t* out) {
  if (!h || !st || (shots && (!variates || !out))) return ALEPH_B200_INVALID_ARGUMENT;
  const size_t sb = sample_scratch_bytes(st->n, ALEPH_B200_SAMPLE_CUMULATIVE, shots);
  const size_t vb = (size_t)shots * 8;
  const size_t need = al(sb) + 2 * al(vb) + 256;
  if (need > kFixedSampleScratchBytes)
    return set_error(h, ALEPH_B200_INVALID_ARGUMENT,
                     "fixed sampling buffer holds %zu bytes; n=%u with %u shots needs %zu (n <= 30 fits up to 65536 shots)",
                     (size_t)kFixedSampleScratchBytes, st->n, shots, need);
  if (int r = bind(h)) return r;
  char* base = nullptr;
  if (int r = fixed_base(h, &base)) return r;
  void* dvar = base + al(sb);
  uint64_t* dout = (uint64_t*)(base + al(sb) + al(vb));
  int32_t* dstatus = (int32_t*)(base + al(sb) + 2 * al(vb));
  // what must start at zero: the status words and the sampler's scratch
  CK(cudaMemsetAsync(dstatus, 0, 64, h->stream), "status clear");
  CK(cudaMemsetAsync(base, 0, sb, h->stream), "scratch clear");
  if (shots) CK(copy_async(h, dvar, variates, vb, cudaMemcpyHostToDevice, h->stream), "variates upload");
  CK(launch_sample(st->amps, st->precision, st->n, shots, ALEPH_B200_SAMPLE_CUMULATIVE, dvar, dout, base, sb, dstatus,
                   h->sm_count, h->stream),
     "sample");
  h->stats.kernel_launches += shots ? 5 : 3;
  int32_t status[4];
  CK(copy_async(h, status, dstatus, 16, cudaMemcpyDeviceToHost, h->stream), "status readback");
  if (shots) CK(copy_async(h, out, dout, vb, cudaMemcpyDeviceToHost, h->stream), "sample readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  count_guard_band(h, st->n, status);
  if (status[0]) {
    aleph_b200_error_info e{};
    e.status = status[0];
    std::snprintf(e.kind, sizeof(e.kind), "state norm2 deviates from 1");
    return report(h, e);
  }
  return ALEPH_B200_OK;
}

int aleph_b200_expectation(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits, const uint8_t* paulis,
                           uint32_t nt, double coefficient, double* out) {
  if (!h || !st || !out || (nt && (!qubits || !paulis))) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  if (int r = ensure(h, h->reduce, (size_t)nb * 3 * 8 + 256)) return r;
  uint64_t xm = 0, zm = 0;
  uint32_t ny = 0;
  bool bad_pauli = false;
  for (uint32_t t = 0; t < nt; ++t) {
    if (qubits[t] >= 64) continue;
    switch (paulis[t]) {
      case ALEPH_PAULI_I: break;
      case ALEPH_PAULI_X: xm |= 1ull << qubits[t]; break;
      case ALEPH_PAULI_Y: xm |= 1ull << qubits[t]; zm |= 1ull << qubits[t]; ++ny; break;
      case ALEPH_PAULI_Z: zm |= 1ull << qubits[t]; break;
      default: bad_pauli = true;
    }
  }
  double* part = (double*)h->reduce.ptr;
  double* out3 = part + 3 * (size_t)nb;
  const bool valid_q = [&] {
    for (uint32_t t = 0; t < nt; ++t)
      if (qubits[t] >= st->n) return false;
    return true;
  }();
  CK(launch_expectation(st->amps, st->precision, st->n, valid_q ? xm : 0, valid_q ? zm : 0, ny, part, nb, out3,
                        h->stream),
     "expectation");
  h->stats.kernel_launches += 2;
  double res[3];
  CK(copy_async(h, res, out3, 24, cudaMemcpyDeviceToHost, h->stream), "expectation readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  // validate_state first (measure.rs:166), then coefficient, then qubits (measure.rs:172-193)
  const double len = (double)(1ull << st->n);
  if (res[1] > 0.0 || !std::isfinite(res[0]) || std::fabs(res[0] - 1.0) > norm_tolerance((uint64_t)len, st->precision)) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_STATE;
    std::snprintf(e.kind, sizeof(e.kind), "state norm2 deviates from 1");
    return report(h, e);
  }
  if (!std::isfinite(coefficient)) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_PAULI_STRING;
    std::snprintf(e.kind, sizeof(e.kind), "non-finite coefficient");
    return report(h, e);
  }
  for (uint32_t t = 0; t < nt; ++t) {
    aleph_b200_error_info e{};
    if (qubits[t] >= st->n) {
      e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
      e.qubit = qubits[t];
      e.num_qubits = st->n;
      return report(h, e);
    }
    for (uint32_t j = 0; j < t; ++j)
      if (qubits[j] == qubits[t]) {
        e.status = ALEPH_B200_DUPLICATE_QUBIT;
        e.qubit = qubits[t];
        return report(h, e);
      }
  }
  if (bad_pauli) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "unknown Pauli code");
  *out = coefficient * res[2];
  return ALEPH_B200_OK;
}

int aleph_b200_expectation_sum(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits,
                               const uint8_t* paulis, const uint64_t* offsets, const double* coefficients,
                               uint64_t n_terms, double* out, double* term_values) {
  if (!h || !st || !out || (n_terms && (!offsets || !coefficients))) return ALEPH_B200_INVALID_ARGUMENT;
  for (uint64_t k = 0; k < n_terms; ++k)
    if (offsets[k + 1] < offsets[k]) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "term offsets decrease");
  if (n_terms && offsets[n_terms] > offsets[0] && (!qubits || !paulis)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  *out = 0.0;
  if (n_terms == 0) return ALEPH_B200_OK;  // the reference's loop evaluates no term and validates nothing

  // per-term masks, as aleph_b200_expectation forms them
  struct TermMasks {
    uint64_t xm = 0, zm = 0;
    uint32_t ny = 0;
    bool bad_pauli = false;
  };
  std::vector<TermMasks> tm(n_terms);
  for (uint64_t k = 0; k < n_terms; ++k) {
    TermMasks& m = tm[k];
    bool in_range = true;
    for (uint64_t t = offsets[k]; t < offsets[k + 1]; ++t) {
      if (qubits[t] >= st->n) in_range = false;
      if (qubits[t] >= 64) continue;
      switch (paulis[t]) {
        case ALEPH_PAULI_I: break;
        case ALEPH_PAULI_X: m.xm |= 1ull << qubits[t]; break;
        case ALEPH_PAULI_Y: m.xm |= 1ull << qubits[t]; m.zm |= 1ull << qubits[t]; ++m.ny; break;
        case ALEPH_PAULI_Z: m.zm |= 1ull << qubits[t]; break;
        default: m.bad_pauli = true;
      }
    }
    if (!in_range) m.xm = m.zm = 0;  // evaluated as the identity; reported as out of range below
  }
  // group the terms by X/Y positions (first appearance order), chunks of MAX_TERMS
  std::vector<PauliGroup> chunks;
  std::vector<std::pair<uint32_t, uint32_t>> slot(n_terms);  // term -> (chunk, index in chunk)
  {
    std::unordered_map<uint64_t, uint32_t> open;  // xmask -> chunk still filling
    for (uint64_t k = 0; k < n_terms; ++k) {
      auto it = open.find(tm[k].xm);
      if (it == open.end() || chunks[it->second].count == (uint32_t)PauliGroup::MAX_TERMS) {
        PauliGroup g{};
        g.xmask = tm[k].xm;
        chunks.push_back(g);
        open[tm[k].xm] = (uint32_t)(chunks.size() - 1);
        it = open.find(tm[k].xm);
      }
      PauliGroup& g = chunks[it->second];
      g.zmask[g.count] = tm[k].zm;
      g.ny[g.count] = tm[k].ny;
      slot[k] = {it->second, g.count};
      ++g.count;
    }
  }
  constexpr size_t NV = 2 + PauliGroup::MAX_TERMS;
  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  if (int r = ensure(h, h->reduce, ((size_t)nb + chunks.size()) * NV * 8 + 256)) return r;
  double* part = (double*)h->reduce.ptr;
  double* res = part + NV * (size_t)nb;
  for (size_t c = 0; c < chunks.size(); ++c)
    CK(launch_pauli_group(st->amps, st->precision, st->n, chunks[c], part, nb, res + NV * c, h->stream),
       "Pauli sum");
  h->stats.kernel_launches += 2 * chunks.size();
  std::vector<double> host(NV * chunks.size());
  CK(copy_async(h, host.data(), res, host.size() * 8, cudaMemcpyDeviceToHost, h->stream), "Pauli sum readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");

  // the reference sums expectation_value over the terms in order
  // (crates/aleph-backend/src/lib.rs:422-432): the state is validated first
  // (measure.rs:166), then each term's coefficient, qubits and duplicates in
  // term order; the first failure is the error
  const double len = (double)(1ull << st->n);
  if (host[1] > 0.0 || !std::isfinite(host[0]) || std::fabs(host[0] - 1.0) > norm_tolerance((uint64_t)len, st->precision)) {
    aleph_b200_error_info e{};
    e.status = ALEPH_B200_INVALID_STATE;
    std::snprintf(e.kind, sizeof(e.kind), "state norm2 deviates from 1");
    return report(h, e);
  }
  double energy = 0.0;
  for (uint64_t k = 0; k < n_terms; ++k) {
    if (!std::isfinite(coefficients[k])) {
      aleph_b200_error_info e{};
      e.status = ALEPH_B200_INVALID_PAULI_STRING;
      std::snprintf(e.kind, sizeof(e.kind), "non-finite coefficient");
      return report(h, e);
    }
    for (uint64_t t = offsets[k]; t < offsets[k + 1]; ++t) {
      aleph_b200_error_info e{};
      if (qubits[t] >= st->n) {
        e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
        e.qubit = qubits[t];
        e.num_qubits = st->n;
        return report(h, e);
      }
      for (uint64_t j = offsets[k]; j < t; ++j)
        if (qubits[j] == qubits[t]) {
          e.status = ALEPH_B200_DUPLICATE_QUBIT;
          e.qubit = qubits[t];
          return report(h, e);
        }
    }
    if (tm[k].bad_pauli) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "unknown Pauli code");
    const double v = coefficients[k] * host[NV * slot[k].first + 2 + slot[k].second];
    if (term_values) term_values[k] = v;
    energy += v;
  }
  *out = energy;
  return ALEPH_B200_OK;
}

int aleph_b200_probabilities(aleph_b200_handle* h, aleph_b200_state* st, const uint32_t* qubits, uint32_t k,
                             double* out) {
  if (!h || !st || !out || (k && !qubits)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  // validate_state first (measure.rs:245)
  if (int r = check_norm_host(h, st, nullptr)) return r;
  for (uint32_t t = 0; t < k; ++t) {
    aleph_b200_error_info e{};
    if (qubits[t] >= st->n) {
      e.status = ALEPH_B200_QUBIT_OUT_OF_RANGE;
      e.qubit = qubits[t];
      e.num_qubits = st->n;
      return report(h, e);
    }
    for (uint32_t j = 0; j < t; ++j)
      if (qubits[j] == qubits[t]) {
        e.status = ALEPH_B200_DUPLICATE_QUBIT;
        e.qubit = qubits[t];
        return report(h, e);
      }
  }
  if (k == 0) {
    out[0] = 1.0;
    return ALEPH_B200_OK;
  }
  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  const size_t dim = (size_t)1 << k;
  const size_t part_bytes = k <= 10 ? (size_t)nb * (dim + 2) * 8 : (size_t)nb * 3 * 8;
  if (int r = ensure(h, h->reduce, part_bytes + 256)) return r;
  if (int r = ensure(h, h->sample, dim * 8 + 256)) return r;
  uint32_t* dq = nullptr;
  CK(cudaMalloc(&dq, 64 * 4), "qubit list");
  cudaError_t e = copy_async(h, dq, qubits, k * 4, cudaMemcpyHostToDevice, h->stream);
  double* dout = (double*)h->sample.ptr;
  double* dnorm = dout + dim;
  if (e == cudaSuccess)
    e = launch_probabilities(st->amps, st->precision, st->n, dq, k, (double*)h->reduce.ptr, nb, dout, dnorm, h->stream);
  if (e == cudaSuccess) e = copy_async(h, out, dout, dim * 8, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dq);
  if (e != cudaSuccess) return cuda_fail(h, e, "probabilities");
  h->stats.kernel_launches += 2;
  return ALEPH_B200_OK;
}

int aleph_b200_get_amplitudes(aleph_b200_handle* h, aleph_b200_state* st, double* out) {
  if (!h || !st || !out) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const uint64_t len = 1ull << st->n;
  if (st->precision == ALEPH_B200_F64) {
    CK(copy_async(h, out, st->amps, st->bytes, cudaMemcpyDeviceToHost, h->stream), "amplitude readback");
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
    return ALEPH_B200_OK;
  }
  std::vector<float> tmp(2 * len);
  CK(copy_async(h, tmp.data(), st->amps, st->bytes, cudaMemcpyDeviceToHost, h->stream), "amplitude readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  for (uint64_t i = 0; i < 2 * len; ++i) out[i] = tmp[i];
  return ALEPH_B200_OK;
}

int aleph_b200_fp64_rate(aleph_b200_handle* h, double* tflops) {
  if (!h || !tflops) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const uint32_t blocks = (uint32_t)h->sm_count * 8, iters = 20000;
  if (int r = ensure(h, h->reduce, (size_t)blocks * 256 * 8 + 256)) return r;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0), "event");
  cudaError_t ce = cudaEventCreate(&e1);
  float best = 0.f;
  for (int k = 0; k < 4 && ce == cudaSuccess; ++k) {  // one warm-up launch, then three timed
    ce = cudaEventRecord(e0, h->stream);
    if (ce == cudaSuccess) ce = launch_dfma_peak((double*)h->reduce.ptr, blocks, iters, h->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(e1, h->stream);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    h->stats.kernel_launches++;
    if (k > 0 && ce == cudaSuccess && (best == 0.f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (ce != cudaSuccess) return cuda_fail(h, ce, "fp64 rate");
  *tflops = 2.0 * dfma_per_launch(blocks, iters) / (best * 1e-3) / 1e12;
  return ALEPH_B200_OK;
}

int aleph_b200_get_amplitude_range(aleph_b200_handle* h, aleph_b200_state* st, uint64_t first, uint64_t count,
                                   double* out) {
  if (!h || !st || (count && !out)) return ALEPH_B200_INVALID_ARGUMENT;
  const uint64_t len = 1ull << st->n;
  if (first > len || count > len - first)
    return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "amplitude window [%llu, +%llu) outside 2^%u",
                     (unsigned long long)first, (unsigned long long)count, st->n);
  if (!count) return ALEPH_B200_OK;
  if (int r = bind(h)) return r;
  if (st->precision == ALEPH_B200_F64) {
    CK(copy_async(h, out, (const char*)st->amps + first * 16, count * 16, cudaMemcpyDeviceToHost, h->stream),
       "amplitude readback");
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
    return ALEPH_B200_OK;
  }
  std::vector<float> tmp(2 * count);
  CK(copy_async(h, tmp.data(), (const char*)st->amps + first * 8, count * 8, cudaMemcpyDeviceToHost, h->stream),
     "amplitude readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  for (uint64_t i = 0; i < 2 * count; ++i) out[i] = tmp[i];
  return ALEPH_B200_OK;
}

int aleph_b200_set_amplitudes(aleph_b200_handle* h, aleph_b200_state* st, const double* in) {
  if (!h || !st || !in) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const uint64_t len = 1ull << st->n;
  if (st->precision == ALEPH_B200_F64) {
    CK(copy_async(h, st->amps, in, st->bytes, cudaMemcpyHostToDevice, h->stream), "amplitude upload");
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
    return ALEPH_B200_OK;
  }
  std::vector<float> tmp(2 * len);
  for (uint64_t i = 0; i < 2 * len; ++i) tmp[i] = (float)in[i];
  CK(copy_async(h, st->amps, tmp.data(), st->bytes, cudaMemcpyHostToDevice, h->stream), "amplitude upload");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  return ALEPH_B200_OK;
}

int aleph_b200_state_memory(aleph_b200_handle* h, aleph_b200_state* st, void** device_ptr, uint64_t* bytes) {
  if (!h || !st || !device_ptr || !bytes) return ALEPH_B200_INVALID_ARGUMENT;
  *device_ptr = st->amps;
  *bytes = st->bytes;
  return ALEPH_B200_OK;
}

int aleph_b200_scale_state(aleph_b200_handle* h, aleph_b200_state* st, double factor) {
  if (!h || !st || !(factor > 0.0) || !std::isfinite(factor)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  if (int r = ensure(h, h->reduce, 256)) return r;
  const double norm2 = 1.0 / (factor * factor);  // the rescale kernel multiplies by 1 / sqrt(norm2)
  CK(copy_async(h, h->reduce.ptr, &norm2, sizeof(norm2), cudaMemcpyHostToDevice, h->stream), "scale upload");
  CK(launch_rescale(st->amps, st->precision, st->n, (const double*)h->reduce.ptr, h->stream), "rescale");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  h->stats.kernel_launches += 1;
  return ALEPH_B200_OK;
}

int aleph_b200_gate_matrix(const aleph_b200_instr* g, const double* matrix_pool, uint64_t pool_len, double* out,
                           int* dim) {
  if (!g || !out || !dim) return ALEPH_B200_INVALID_ARGUMENT;
  aleph_b200_error_info e{};
  return gate_matrix_dense(*g, matrix_pool, pool_len, out, dim, &e);
}

int aleph_b200_norm_sqr(aleph_b200_handle* h, aleph_b200_state* st, double* out) {
  if (!h || !st || !out) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const uint32_t nb = reduce_blocks(st->n, h->sm_count);
  if (int r = ensure(h, h->reduce, (size_t)nb * 3 * 8 + 256)) return r;
  double* part = (double*)h->reduce.ptr;
  double* out2 = part + 3 * (size_t)nb;
  CK(launch_norm(st->amps, st->precision, st->n, part, nb, out2, h->stream), "norm");
  h->stats.kernel_launches += 2;
  double res[2];
  CK(copy_async(h, res, out2, 16, cudaMemcpyDeviceToHost, h->stream), "norm readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  *out = res[1] > 0.0 ? NAN : res[0];
  return ALEPH_B200_OK;
}

int aleph_b200_get_stream(const aleph_b200_handle* h, void** stream) {
  if (!h || !stream) return ALEPH_B200_INVALID_ARGUMENT;
  *stream = (void*)h->stream;
  return ALEPH_B200_OK;
}

int aleph_b200_synchronize(aleph_b200_handle* h) {
  if (!h) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  return ALEPH_B200_OK;
}

int aleph_b200_last_error(const aleph_b200_handle* h, char* buf, uint64_t len) {
  if (!h || !buf || !len) return ALEPH_B200_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", h->err_msg.c_str());
  return h->err.status;
}

int aleph_b200_last_error_info(const aleph_b200_handle* h, aleph_b200_error_info* out) {
  if (!h || !out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = h->err;
  return h->err.status;
}

int aleph_b200_set_tuning(aleph_b200_handle* h, const char* key, int64_t value) {
  if (!h || !key) return ALEPH_B200_INVALID_ARGUMENT;
  if (!std::strcmp(key, "tile_r")) {
    if (value < 1 || value > 5) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "tile_r must be in 1..5");
    h->opts.tile_r = (uint32_t)value;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "record_passes")) {
    h->record_passes = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "tile_occupancy")) {
    if (value != 0 && (value < 2 || value > 4))
      return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "tile_occupancy must be 0 or in 2..4");
    h->opts.tile_occupancy = (uint32_t)value;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "renormalize")) {
    h->opts.renormalize = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "pair_fusion")) {
    h->opts.pair_fusion = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "tensor_blocks")) {
    if (h->precision != ALEPH_B200_TC32)
      return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "tensor_blocks applies to TC32 handles only");
    h->opts.tensor_blocks = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "block_window_search")) {
    h->opts.block_window_search = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "smem_max_n")) {
    if (value < 0 || value > 12) return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "smem_max_n must be in 0..12");
    h->opts.smem_max_n = (uint32_t)value;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "relabel_swaps")) {
    h->opts.relabel_swaps = value != 0;
    return ALEPH_B200_OK;
  }
  if (!std::strcmp(key, "paged_local_qubits")) {
    if (value < 0 || value > (int64_t)kMaxQubits)
      return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "paged_local_qubits must be in 0..%u", kMaxQubits);
    h->paged_local_max = (uint32_t)value;
    return ALEPH_B200_OK;
  }
  return set_error(h, ALEPH_B200_INVALID_ARGUMENT, "unknown tuning key %s", key);
}

int aleph_b200_describe_plan(uint32_t num_qubits, const aleph_b200_plan_config* config, const aleph_b200_instr* in,
                             uint64_t count, const aleph_b200_pools* pools, aleph_b200_pass_record* out, uint64_t cap,
                             uint64_t* n_passes) {
  if (!config || !n_passes || (!in && count) || (cap && !out)) return ALEPH_B200_INVALID_ARGUMENT;
  if (config->precision < ALEPH_B200_F64 || config->precision > ALEPH_B200_TC32 || config->tile_r < 1 ||
      config->tile_r > 5 || config->smem_max_n > 12 || num_qubits > 40 ||
      (config->tile_occupancy != 0 && (config->tile_occupancy < 2 || config->tile_occupancy > 4)))
    return ALEPH_B200_INVALID_ARGUMENT;
  FullHandle tmp;  // host-only: validation messages land here, no device is touched
  tmp.opts.tile_r = config->tile_r;
  tmp.opts.smem_max_n = config->smem_max_n;
  tmp.opts.tensor_blocks = config->precision == ALEPH_B200_TC32;
  tmp.opts.block_window_search = config->block_window_search != 0;
  tmp.opts.tile_occupancy = config->tile_occupancy;
  tmp.opts.relabel_swaps = config->keep_swaps == 0;
  tmp.opts.pair_fusion = config->no_pair_fusion == 0;
  std::vector<Lowered> ops;
  if (int r = lower_stream(&tmp, num_qubits, in, count, pools, &ops)) return r;
  Plan P;
  if (int s = build_plan(ops, num_qubits, tmp.opts, &P)) return s;
  const double bpa = config->precision == ALEPH_B200_F64 ? 16.0 : 8.0;
  const double len = (double)(1ull << num_qubits);
  *n_passes = P.passes.size();
  for (size_t k = 0; k < P.passes.size() && k < cap; ++k) {
    const Pass& ps = P.passes[k];
    aleph_b200_pass_record r{};
    r.kind = (uint32_t)ps.kind;
    r.gates = ps.gates;
    r.n = num_qubits;
    const uint32_t* qs = ps.kind == PASS_BLOCK ? ps.block.bq : ps.tile.hq;
    r.nq = ps.kind == PASS_BLOCK ? 6 : ps.kind == PASS_TILE ? ps.tile.R : 0;
    for (uint32_t j = 0; j < r.nq && j < 8; ++j) r.qubits[j] = qs[j];
    r.post_ops = ps.kind == PASS_BLOCK ? ps.block.post_count : 0;
    r.lane_ops = ps.lane_ops;
    r.dense_ops = ps.dense_ops;
    r.diag_ops = ps.diag_ops;
    r.fma_per_amp = ps.fma_per_amp;
    r.variant = ps.kind == PASS_TILE ? ps.tile.occupancy : 0;
    r.bytes = (ps.kind == PASS_MEASURE ? 3 : 2) * len * bpa;
    out[k] = r;
  }
  return ALEPH_B200_OK;
}

int aleph_b200_get_pass_records(const aleph_b200_handle* h, aleph_b200_pass_record* out, uint64_t cap, uint64_t* n) {
  if (!h || !n || (cap && !out)) return ALEPH_B200_INVALID_ARGUMENT;
  *n = h->records.size();
  for (size_t i = 0; i < h->records.size() && i < cap; ++i) out[i] = h->records[i];
  return ALEPH_B200_OK;
}

int aleph_b200_get_stats(const aleph_b200_handle* h, aleph_b200_stats* out) {
  if (!h || !out) return ALEPH_B200_INVALID_ARGUMENT;
  *out = h->stats;
  return ALEPH_B200_OK;
}

int aleph_b200_reset_stats(aleph_b200_handle* h) {
  if (!h) return ALEPH_B200_INVALID_ARGUMENT;
  h->stats = aleph_b200_stats{};
  return ALEPH_B200_OK;
}

// ---- the learned planner's cost model (kernels_mlp.cu) -------------------------
struct aleph_b200_mlp {
  int F = 0, H = 0;
  size_t np = 0;
  Scratch params, grads, adam_m, adam_v;  // np floats each
  Scratch work;                           // X | y | activations | backward scratch | loss
  int step = 0;
};

namespace {
// Work region for a batch of B samples: X (B F) | y (B) | acts (3 B H + B) | dbuf (2 B H) | loss.
size_t mlp_work_floats(int B, int F, int H) {
  return (size_t)B * F + B + (size_t)3 * B * H + B + (size_t)2 * B * H + 4;
}
int mlp_upload_batch(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, const float* y, int B) {
  if (int r = ensure(h, m->work, mlp_work_floats(B, m->F, m->H) * 4)) return r;
  float* w = (float*)m->work.ptr;
  CK(copy_async(h, w, X, (size_t)B * m->F * 4, cudaMemcpyHostToDevice, h->stream), "mlp batch upload");
  if (y) CK(copy_async(h, w + (size_t)B * m->F, y, (size_t)B * 4, cudaMemcpyHostToDevice, h->stream), "mlp target upload");
  return 0;
}
}  // namespace

int aleph_b200_mlp_create(aleph_b200_handle* h, uint32_t n_features, uint32_t hidden, uint64_t seed,
                          aleph_b200_mlp** out) {
  if (!h || !out || n_features == 0 || n_features > 1024 || hidden == 0 || hidden > 1024)
    return ALEPH_B200_INVALID_ARGUMENT;
  *out = nullptr;
  if (int r = bind(h)) return r;
  aleph_b200_mlp* m = new (std::nothrow) aleph_b200_mlp();
  if (!m) return set_error(h, ALEPH_B200_DEVICE_FAILURE, "host allocation failed");
  m->F = (int)n_features;
  m->H = (int)hidden;
  m->np = mlp_param_count(m->F, m->H);
  // He-uniform weights (bound sqrt(6 / fan_in)), zero biases, from a splitmix64 stream
  std::vector<float> p(m->np, 0.f);
  uint64_t x = seed;
  const int ins[4] = {m->F, m->H, m->H, m->H}, outs[4] = {m->H, m->H, m->H, 1};
  size_t off = 0;
  for (int l = 0; l < 4; ++l) {
    const float bound = std::sqrt(6.f / (float)ins[l]);
    for (size_t k = 0; k < (size_t)ins[l] * outs[l]; ++k) {
      const double u = (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0);
      p[off + k] = (float)((2.0 * u - 1.0) * bound);
    }
    off += (size_t)ins[l] * outs[l] + outs[l];
  }
  int r = ensure(h, m->params, m->np * 4);
  if (!r) r = ensure(h, m->grads, m->np * 4);
  if (!r) r = ensure(h, m->adam_m, m->np * 4);
  if (!r) r = ensure(h, m->adam_v, m->np * 4);
  if (r) {
    for (Scratch* s : {&m->params, &m->grads, &m->adam_m, &m->adam_v})
      if (s->ptr) cudaFree(s->ptr);
    delete m;
    return r;
  }
  cudaError_t e = copy_async(h, m->params.ptr, p.data(), m->np * 4, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->adam_m.ptr, 0, m->np * 4, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->adam_v.ptr, 0, m->np * 4, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    for (Scratch* s : {&m->params, &m->grads, &m->adam_m, &m->adam_v})
      if (s->ptr) cudaFree(s->ptr);
    delete m;
    return cuda_fail(h, e, "mlp init");
  }
  *out = m;
  return ALEPH_B200_OK;
}

int aleph_b200_mlp_free(aleph_b200_handle* h, aleph_b200_mlp* m) {
  if (!m) return ALEPH_B200_OK;
  if (h) {
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
  }
  for (Scratch* s : {&m->params, &m->grads, &m->adam_m, &m->adam_v, &m->work})
    if (s->ptr) cudaFree(s->ptr);
  delete m;
  return ALEPH_B200_OK;
}

int aleph_b200_mlp_params(aleph_b200_handle* h, aleph_b200_mlp* m, float* get, const float* set, uint64_t* count) {
  if (!h || !m) return ALEPH_B200_INVALID_ARGUMENT;
  if (count) *count = m->np;
  if (int r = bind(h)) return r;
  if (set) {
    CK(copy_async(h, m->params.ptr, set, m->np * 4, cudaMemcpyHostToDevice, h->stream), "mlp params upload");
    CK(cudaMemsetAsync(m->adam_m.ptr, 0, m->np * 4, h->stream), "adam reset");
    CK(cudaMemsetAsync(m->adam_v.ptr, 0, m->np * 4, h->stream), "adam reset");
    m->step = 0;
  }
  if (get) CK(copy_async(h, get, m->params.ptr, m->np * 4, cudaMemcpyDeviceToHost, h->stream), "mlp params readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  return ALEPH_B200_OK;
}

int aleph_b200_mlp_predict(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, uint32_t n, float* y_out) {
  if (!h || !m || (n && (!X || !y_out))) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const int F = m->F, H = m->H;
  for (uint32_t b0 = 0; b0 < n; b0 += 4096) {
    const int B = (int)std::min<uint32_t>(4096, n - b0);
    if (int r = mlp_upload_batch(h, m, X + (size_t)b0 * F, nullptr, B)) return r;
    float* w = (float*)m->work.ptr;
    float* acts = w + (size_t)B * F + B;
    CK(mlp_forward((const float*)m->params.ptr, w, acts, B, F, H, h->stream), "mlp forward");
    CK(copy_async(h, y_out + b0, acts + (size_t)3 * B * H, (size_t)B * 4, cudaMemcpyDeviceToHost, h->stream),
       "mlp readback");
    CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  }
  h->stats.kernel_launches += 4;
  return ALEPH_B200_OK;
}

int aleph_b200_mlp_gradients(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, const float* y, uint32_t n,
                             float* grads_out, float* loss_out) {
  if (!h || !m || !X || !y || !n || n > 65536) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const int F = m->F, H = m->H, B = (int)n;
  if (int r = mlp_upload_batch(h, m, X, y, B)) return r;
  float* w = (float*)m->work.ptr;
  float* acts = w + (size_t)B * F + B;
  float* dbuf = acts + (size_t)3 * B * H + B;
  float* loss = dbuf + (size_t)2 * B * H;
  CK(mlp_forward((const float*)m->params.ptr, w, acts, B, F, H, h->stream), "mlp forward");
  CK(mlp_backward((const float*)m->params.ptr, w, acts, w + (size_t)B * F, (float*)m->grads.ptr, dbuf, loss, B, F, H,
                  h->stream),
     "mlp backward");
  if (grads_out) CK(copy_async(h, grads_out, m->grads.ptr, m->np * 4, cudaMemcpyDeviceToHost, h->stream), "grad readback");
  if (loss_out) CK(copy_async(h, loss_out, loss, 4, cudaMemcpyDeviceToHost, h->stream), "loss readback");
  CK(cudaStreamSynchronize(h->stream), "stream synchronize");
  return ALEPH_B200_OK;
}

int aleph_b200_mlp_train(aleph_b200_handle* h, aleph_b200_mlp* m, const float* X, const float* y, uint32_t n,
                         uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* final_loss) {
  if (!h || !m || !X || !y || !n || !batch || batch > 65536 || !(lr > 0.f)) return ALEPH_B200_INVALID_ARGUMENT;
  if (int r = bind(h)) return r;
  const int F = m->F, H = m->H;
  const int B = (int)std::min<uint32_t>(batch, n);
  // the whole data set lives on the device, reshuffled on the host once per epoch
  Scratch data;
  if (int r = ensure(h, data, (size_t)n * (F + 1) * 4)) return r;
  if (int r = ensure(h, m->work, mlp_work_floats(B, F, H) * 4)) {
    cudaFree(data.ptr);
    return r;
  }
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  std::vector<float> hx((size_t)n * F), hy(n);
  uint64_t rs = seed;
  float* dX = (float*)data.ptr;
  float* dY = dX + (size_t)n * F;
  float* w = (float*)m->work.ptr;
  float* acts = w + (size_t)B * F + B;
  float* dbuf = acts + (size_t)3 * B * H + B;
  float* loss = dbuf + (size_t)2 * B * H;
  float last = 0.f;
  cudaError_t e = cudaSuccess;
  for (uint32_t ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix64(rs) % (i + 1)]);  // Fisher-Yates
    for (uint32_t i = 0; i < n; ++i) {
      std::memcpy(&hx[(size_t)i * F], X + (size_t)perm[i] * F, (size_t)F * 4);
      hy[i] = y[perm[i]];
    }
    e = copy_async(h, dX, hx.data(), hx.size() * 4, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = copy_async(h, dY, hy.data(), hy.size() * 4, cudaMemcpyHostToDevice, h->stream);
    for (uint32_t b0 = 0; b0 + (uint32_t)B <= n && e == cudaSuccess; b0 += B) {
      const float* xb = dX + (size_t)b0 * F;
      const float* yb = dY + b0;
      e = mlp_forward((const float*)m->params.ptr, xb, acts, B, F, H, h->stream);
      if (e == cudaSuccess)
        e = mlp_backward((const float*)m->params.ptr, xb, acts, yb, (float*)m->grads.ptr, dbuf, loss, B, F, H,
                         h->stream);
      if (e == cudaSuccess)
        e = mlp_adam((float*)m->params.ptr, (const float*)m->grads.ptr, (float*)m->adam_m.ptr, (float*)m->adam_v.ptr,
                     m->np, lr, ++m->step, h->stream);
      h->stats.kernel_launches += 16;
    }
    // every epoch's host data is staged before the next shuffle overwrites it
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  }
  if (e == cudaSuccess) e = copy_async(h, &last, loss, 4, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(data.ptr);
  if (e != cudaSuccess) return cuda_fail(h, e, "mlp training");
  if (final_loss) *final_loss = last;
  return ALEPH_B200_OK;
}

}  // extern "C"
