// common.cuh — device helpers shared by the engine's kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "engine.h"

namespace ab {

template <typename Real>
struct V2T;
template <>
struct V2T<double> {
  using type = double2;
};
template <>
struct V2T<float> {
  using type = float2;
};
template <typename Real>
using V2 = typename V2T<Real>::type;

template <typename Real>
__device__ __forceinline__ V2<Real> mk(Real x, Real y) {
  V2<Real> r;
  r.x = x;
  r.y = y;
  return r;
}
template <typename Real>
__device__ __forceinline__ V2<Real> cmul(V2<Real> a, V2<Real> b) {
  return mk<Real>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c*d
template <typename Real>
__device__ __forceinline__ V2<Real> cmul2(V2<Real> a, V2<Real> b, V2<Real> c, V2<Real> d) {
  return mk<Real>(a.x * b.x - a.y * b.y + c.x * d.x - c.y * d.y, a.x * b.y + a.y * b.x + c.x * d.y + c.y * d.x);
}
template <typename Real>
__device__ __forceinline__ V2<Real> cadd(V2<Real> a, V2<Real> b) {
  return mk<Real>(a.x + b.x, a.y + b.y);
}
template <typename Real>
__device__ __forceinline__ V2<Real> cneg(V2<Real> a) {
  return mk<Real>(-a.x, -a.y);
}

template <typename Real>
__device__ __forceinline__ V2<Real> ld_amp(const V2<Real>* p) {
  return __ldcg(p);
}
template <typename Real>
__device__ __forceinline__ void st_amp(V2<Real>* p, V2<Real> v) {
  __stcg(p, v);
}

template <typename Real>
__device__ __forceinline__ V2<Real> ld_coef(const V2<Real>* p) {
  return __ldg(p);
}

template <typename Real>
__device__ __forceinline__ V2<Real> shfl_xor(V2<Real> v, int m) {
  V2<Real> r;
  r.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  r.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  return r;
}

// Phase of a DiagonalPhase polynomial at basis index x
// (crates/aleph-sv/src/kernels/diagonal_phase.rs:26-41): sum of the angles
// of the terms whose every condition mask has odd parity with x.
__device__ __forceinline__ double poly_phase(const PolyTables& t, uint32_t first, uint32_t count, uint64_t x) {
  double phi = 0.0;
  for (uint32_t i = first; i < first + count; ++i) {
    const uint32_t off = __ldg(&t.cond_off[i]);
    const uint32_t cnt = __ldg(&t.cond_cnt[i]);
    bool all = true;
    for (uint32_t c = 0; c < cnt; ++c)
      if ((__popcll(__ldg(&t.conds[off + c]) & x) & 1) == 0) {
        all = false;
        break;
      }
    if (all) phi += __ldg(&t.angle[i]);
  }
  return phi;
}

// Apply one diagonal op to an amplitude at global index g.
template <typename Real>
__device__ __forceinline__ V2<Real> apply_diag_op(const Op& op, V2<Real> a, uint64_t g, const V2<Real>* coef,
                                                  const PolyTables& poly) {
  if ((g & op.ctrl) != op.ctrl) return a;
  switch (op.type) {
    case OP_NEG:
      return ((g & op.mask) == op.mask) ? cneg<Real>(a) : a;
    case OP_CPHASE:
      return ((g & op.mask) == op.mask) ? cmul<Real>(ld_coef<Real>(coef + op.coef), a) : a;
    case OP_DIAG: {
      uint32_t idx = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
        if (i < op.nq) idx = (idx << 1) | (uint32_t)((g >> op.q[i]) & 1);
      return cmul<Real>(ld_coef<Real>(coef + op.coef + idx), a);
    }
    case OP_POLY: {
      const double phi = poly_phase(poly, (uint32_t)op.mask, op.aux, g);
      double s, c;
      sincos(phi, &s, &c);
      return mk<Real>((Real)((double)a.x * c - (double)a.y * s), (Real)((double)a.x * s + (double)a.y * c));
    }
  }
  return a;
}

__device__ __forceinline__ bool is_diag_type(uint8_t t) {
  return t == OP_NEG || t == OP_CPHASE || t == OP_DIAG || t == OP_POLY;
}

// Insert a zero bit at position `pos` of x.
__device__ __forceinline__ uint64_t insert_zero(uint64_t x, uint32_t pos) {
  const uint64_t lo = x & ((1ull << pos) - 1);
  return ((x >> pos) << (pos + 1)) | lo;
}

// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Deadline of every bounded wait: a pipeline stage that has not completed
// within this time is treated as stuck, and the kernel reports an error.
constexpr uint64_t kWaitDeadlineNs = 1000000000ull;  // 1 s

// ---- mbarriers and bulk-async copies (shared by the pipelined kernels) ------
namespace async {
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
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
// Wait for the phase with the given parity, bounded by kWaitDeadlineNs of
// wall time (not by an iteration count: one try_wait may itself suspend the
// thread for a while). Returns false on expiry, or once *abort_flag is set
// by another role of the kernel (polled every 256 tries).
__device__ __forceinline__ bool mbar_wait_deadline(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (globaltimer_ns() - t0 > kWaitDeadlineNs) return false;
    }
  }
}
// Non-multicast bulk copy global -> shared, completing on an mbarrier.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
// Orders this thread's generic shared-memory accesses before later async-proxy ones.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
}  // namespace async

}  // namespace ab
