// kernels_readout.cu — on-device FP64 readout: norm, measurement
// (reduce + decide + collapse, no host round trip), Pauli expectation and
// marginal probabilities. All reductions accumulate in FP64 (also for FP32
// states) and are deterministic: fixed per-block partials, then one block
// sums the partials in index order.
//
// Semantics: validate_state (crates/aleph-sv/src/measure.rs:23-33,
// crates/aleph-sv/src/sampling.rs:36-57), measure_impl (measure.rs:41-102),
// expectation_value_impl (measure.rs:155-233), probabilities_impl
// (measure.rs:239-273).

#include <cmath>

#include "common.cuh"

namespace ab {

constexpr int RB = 256;  // threads per reduction block

uint32_t reduce_blocks(uint32_t n, int sm_count) {
  const uint64_t len = 1ull << n;
  uint64_t b = (len + RB * 8 - 1) / (RB * 8);
  const uint64_t cap = (uint64_t)sm_count * 8;
  if (b > cap) b = cap;
  return (uint32_t)(b ? b : 1);
}

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out) {
  __shared__ double red[NV][RB / 32];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
    for (int o = 16; o; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < RB / 32; ++w) s += red[k][w];
      out[k] = s;
    }
  }
}

// partials[b*NV + k] -> out[k], summed in block order by one thread.
template <int NV>
__global__ void finish_kernel(const double* __restrict__ partials, uint32_t nblocks, double* __restrict__ out) {
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (uint32_t b = 0; b < nblocks; ++b) s += partials[(size_t)b * NV + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

template <typename Real>
__device__ __forceinline__ double abs2(V2<Real> a) {
  const double x = a.x, y = a.y;
  return x * x + y * y;
}

// ---- norm: [sum |a|^2, non-finite count] ------------------------------------
template <typename Real>
__global__ void __launch_bounds__(RB) norm_kernel(const V2<Real>* __restrict__ amps, uint64_t len,
                                                  double* __restrict__ partials) {
  double v[2] = {0.0, 0.0};
  // four independent loads per step keep enough bytes in flight for the
  // 8-byte complex64 amplitudes (one load per step left the pass latency-bound)
  const uint64_t stride = (uint64_t)gridDim.x * RB;
  uint64_t i = (uint64_t)blockIdx.x * RB + threadIdx.x;
  for (; i + 3 * stride < len; i += 4 * stride) {
    V2<Real> a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = ld_amp<Real>(amps + i + k * stride);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double p = abs2<Real>(a[k]);
      if (isfinite(p)) v[0] += p;
      else v[1] += 1.0;
    }
  }
  for (; i < len; i += stride) {
    const double p = abs2<Real>(ld_amp<Real>(amps + i));
    if (isfinite(p)) v[0] += p;
    else v[1] += 1.0;
  }
  block_reduce_store<2>(v, partials + 2 * blockIdx.x);
}

cudaError_t launch_norm(const void* amps, int precision, uint32_t n, double* partials, uint32_t nblocks, double* out2,
                        cudaStream_t s) {
  const uint64_t len = 1ull << n;
  if (precision == ALEPH_B200_F64) norm_kernel<double><<<nblocks, RB, 0, s>>>((const double2*)amps, len, partials);
  else norm_kernel<float><<<nblocks, RB, 0, s>>>((const float2*)amps, len, partials);
  finish_kernel<2><<<1, 32, 0, s>>>(partials, nblocks, out2);
  return cudaGetLastError();
}

// ---- measurement ---------------------------------------------------------------
// [p0, p1, non-finite count]
template <typename Real>
__global__ void __launch_bounds__(RB) branch_kernel(const V2<Real>* __restrict__ amps, uint64_t len, uint64_t qb,
                                                    double* __restrict__ partials) {
  double v[3] = {0.0, 0.0, 0.0};
  auto add = [&](uint64_t i, double p) {
    if (!isfinite(p)) v[2] += 1.0;
    else if (i & qb) v[1] += p;
    else v[0] += p;
  };
  const uint64_t stride = (uint64_t)gridDim.x * RB;
  uint64_t i = (uint64_t)blockIdx.x * RB + threadIdx.x;
  for (; i + 3 * stride < len; i += 4 * stride) {  // four loads in flight per step (see norm_kernel)
    V2<Real> a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) a[k] = ld_amp<Real>(amps + i + k * stride);
#pragma unroll
    for (int k = 0; k < 4; ++k) add(i + k * stride, abs2<Real>(a[k]));
  }
  for (; i < len; i += stride) add(i, abs2<Real>(ld_amp<Real>(amps + i)));
  block_reduce_store<3>(v, partials + 3 * blockIdx.x);
}

// status[0]: error code (0 ok), status[1]: uniforms consumed, status[2]: failing qubit;
// dec[0] = outcome (0/1), dec[1] = 1/norm scale; dval[0] = reported probability.
__global__ void measure_decide_kernel(const double* __restrict__ sums, uint32_t qubit, uint64_t len,
                                      const double* __restrict__ uniforms, uint32_t n_uniforms, int32_t* status,
                                      double* dec, uint8_t* outcome_slot, double tol) {
  if (threadIdx.x != 0) return;
  dec[0] = -1.0;  // "skip collapse" unless a decision is made below
  if (status[0] != 0) return;  // an earlier instruction failed: do nothing further
  const double p0r = sums[0], p1r = sums[1], bad = sums[2];
  const double total = p0r + p1r;
  if (bad > 0.0 || !isfinite(total) || fabs(total - 1.0) > tol) {
    status[0] = ALEPH_B200_INVALID_STATE;
    status[2] = (int32_t)qubit;
    return;
  }
  const double p0 = fmin(fmax(p0r, 0.0), 1.0), p1 = fmin(fmax(p1r, 0.0), 1.0);
  const bool one_degen = p1 < 1e-300, zero_degen = p0 < 1e-300;
  bool outcome;
  double p;
  if (zero_degen && one_degen) {
    status[0] = ALEPH_B200_DEGENERATE_MEASUREMENT;
    status[2] = (int32_t)qubit;
    dec[2] = fmax(p1, p0);
    return;
  } else if (zero_degen) {
    outcome = true;
    p = p1;
  } else if (one_degen) {
    outcome = false;
    p = p0;
  } else {
    const uint32_t used = (uint32_t)status[1];
    if (used >= n_uniforms) {
      status[0] = ALEPH_B200_INVALID_ARGUMENT;
      status[2] = (int32_t)qubit;
      return;
    }
    outcome = uniforms[used] < p1;
    status[1] = (int32_t)(used + 1);
    p = outcome ? p1 : p0;
  }
  dec[0] = outcome ? 1.0 : 0.0;
  dec[1] = sqrt(p);
  if (outcome_slot) *outcome_slot = outcome ? 1 : 0;
}

template <typename Real>
__global__ void collapse_kernel(V2<Real>* __restrict__ amps, uint64_t len, uint64_t qb, const double* __restrict__ dec) {
  const double o = dec[0];
  if (o < 0.0) return;
  const bool outcome = o > 0.5;
  const double norm = dec[1];
  const double d = norm * norm;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const bool bit = (i & qb) != 0;
    V2<Real> a = ld_amp<Real>(amps + i);
    if (bit == outcome) {
      // num-complex division by Complex::new(norm, 0.0), as the reference's `*a /= ...`
      a = mk<Real>((Real)(((double)a.x * norm) / d), (Real)(((double)a.y * norm) / d));
    } else {
      a = mk<Real>(0, 0);
    }
    st_amp<Real>(amps + i, a);
  }
}

cudaError_t launch_measure_pass(void* amps, int precision, uint32_t n, uint32_t qubit, double* partials,
                                uint32_t nblocks, const double* uniforms, uint32_t n_uniforms, int32_t* status,
                                uint8_t* outcome_slot, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  const uint64_t qb = 1ull << qubit;
  double* sums = partials + 3 * (size_t)nblocks;
  double* dec = sums + 4;
  if (precision == ALEPH_B200_F64) branch_kernel<double><<<nblocks, RB, 0, s>>>((const double2*)amps, len, qb, partials);
  else branch_kernel<float><<<nblocks, RB, 0, s>>>((const float2*)amps, len, qb, partials);
  finish_kernel<3><<<1, 32, 0, s>>>(partials, nblocks, sums);
  measure_decide_kernel<<<1, 32, 0, s>>>(sums, qubit, len, uniforms, n_uniforms, status, dec, outcome_slot,
                                         norm_tolerance(len, precision));
  const uint64_t b = (len + 255) / 256;
  const unsigned blocks = (unsigned)(b > 148ull * 32 ? 148ull * 32 : b);
  if (precision == ALEPH_B200_F64) collapse_kernel<double><<<blocks, 256, 0, s>>>((double2*)amps, len, qb, dec);
  else collapse_kernel<float><<<blocks, 256, 0, s>>>((float2*)amps, len, qb, dec);
  return cudaGetLastError();
}

// ---- Pauli expectation: [sum |a|^2, non-finite count, Re <psi|P|psi>] ----------
// P = (x) Paulis with X/Y positions `xmask` (flip), Z/Y positions `zmask`
// (sign), ny = number of Y factors. (P psi)_i = i^ny (-1)^{popc(zmask & j)} psi_j
// with j = i ^ xmask: Y = i X Z, X flips, Z signs the pre-image bit.
template <typename Real>
__global__ void __launch_bounds__(RB) expect_kernel(const V2<Real>* __restrict__ amps, uint64_t len, uint64_t xmask,
                                                    uint64_t zmask, uint32_t ny, double* __restrict__ partials) {
  double v[3] = {0.0, 0.0, 0.0};
  for (uint64_t i = (uint64_t)blockIdx.x * RB + threadIdx.x; i < len; i += (uint64_t)gridDim.x * RB) {
    const V2<Real> a = ld_amp<Real>(amps + i);
    const double p = abs2<Real>(a);
    if (!isfinite(p)) {
      v[1] += 1.0;
      continue;
    }
    v[0] += p;
    const uint64_t j = i ^ xmask;
    const V2<Real> b = (xmask == 0) ? a : ld_amp<Real>(amps + j);
    // conj(a) * b
    double re = (double)a.x * b.x + (double)a.y * b.y;
    double im = (double)a.x * b.y - (double)a.y * b.x;
    if (__popcll(zmask & j) & 1) {
      re = -re;
      im = -im;
    }
    // multiply by i^ny and keep the real part
    switch (ny & 3) {
      case 0: v[2] += re; break;
      case 1: v[2] += -im; break;
      case 2: v[2] += -re; break;
      default: v[2] += im; break;
    }
  }
  block_reduce_store<3>(v, partials + 3 * blockIdx.x);
}

cudaError_t launch_expectation(const void* amps, int precision, uint32_t n, uint64_t xmask, uint64_t zmask,
                               uint32_t ny, double* partials, uint32_t nblocks, double* out3, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  if (precision == ALEPH_B200_F64)
    expect_kernel<double><<<nblocks, RB, 0, s>>>((const double2*)amps, len, xmask, zmask, ny, partials);
  else
    expect_kernel<float><<<nblocks, RB, 0, s>>>((const float2*)amps, len, xmask, zmask, ny, partials);
  finish_kernel<3><<<1, 32, 0, s>>>(partials, nblocks, out3);
  return cudaGetLastError();
}

// ---- Pauli sum: up to 16 terms that share one X/Y (flip) mask, one sweep ----------
// For every term: Re <psi|P|psi> with P as in expect_kernel. (P psi)_i differs
// between the terms of a group only in the sign (-1)^{popc(zmask & j)} and the
// factor i^ny, so conj(a_i) a_j is formed once per amplitude and shared.
// partials per block: [sum |a|^2, non-finite count, term 0 .. 15].
template <typename Real, bool DIAG>
__global__ void __launch_bounds__(RB) pauli_group_kernel(const V2<Real>* __restrict__ amps, uint64_t len,
                                                         const PauliGroup g, double* __restrict__ partials) {
  double v[2 + PauliGroup::MAX_TERMS];
#pragma unroll
  for (int k = 0; k < 2 + PauliGroup::MAX_TERMS; ++k) v[k] = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * RB;
  uint64_t i0 = (uint64_t)blockIdx.x * RB + threadIdx.x;
  if constexpr (DIAG) {  // no X/Y factor: Re conj(a) a = |a|^2 and ny = 0
    auto add = [&](uint64_t i, double p) {
      if (!isfinite(p)) {
        v[1] += 1.0;
        return;
      }
      v[0] += p;
#pragma unroll
      for (int k = 0; k < PauliGroup::MAX_TERMS; ++k)
        if (k < (int)g.count) v[2 + k] += (__popcll(g.zmask[k] & i) & 1) ? -p : p;
    };
    for (; i0 + 3 * stride < len; i0 += 4 * stride) {  // four loads in flight per step (see norm_kernel)
      V2<Real> a[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = ld_amp<Real>(amps + i0 + k * stride);
#pragma unroll
      for (int k = 0; k < 4; ++k) add(i0 + k * stride, abs2<Real>(a[k]));
    }
  }
  for (uint64_t i = i0; i < len; i += stride) {
    const V2<Real> a = ld_amp<Real>(amps + i);
    const double p = abs2<Real>(a);
    if (!isfinite(p)) {
      v[1] += 1.0;
      continue;
    }
    v[0] += p;
    if constexpr (DIAG) {
#pragma unroll
      for (int k = 0; k < PauliGroup::MAX_TERMS; ++k)
        if (k < (int)g.count) v[2 + k] += (__popcll(g.zmask[k] & i) & 1) ? -p : p;
    } else {
      const uint64_t j = i ^ g.xmask;
      const V2<Real> b = ld_amp<Real>(amps + j);
      const double re = (double)a.x * b.x + (double)a.y * b.y;  // conj(a) * b
      const double im = (double)a.x * b.y - (double)a.y * b.x;
#pragma unroll
      for (int k = 0; k < PauliGroup::MAX_TERMS; ++k)
        if (k < (int)g.count) {
          // i^ny: ny & 3 = 0, 1, 2, 3 keeps re, -im, -re, im
          const uint32_t q = g.ny[k] & 3;
          double t = (q & 1) ? im : re;
          if ((q == 1 || q == 2) != (bool)(__popcll(g.zmask[k] & j) & 1)) t = -t;
          v[2 + k] += t;
        }
    }
  }
  block_reduce_store<2 + PauliGroup::MAX_TERMS>(v, partials + (2 + PauliGroup::MAX_TERMS) * (size_t)blockIdx.x);
}

cudaError_t launch_pauli_group(const void* amps, int precision, uint32_t n, const PauliGroup& g, double* partials,
                               uint32_t nblocks, double* out, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  constexpr int NV = 2 + PauliGroup::MAX_TERMS;
  if (g.count == 0 || g.count > (uint32_t)PauliGroup::MAX_TERMS) return cudaErrorInvalidValue;
  const bool diag = g.xmask == 0;
  if (precision == ALEPH_B200_F64) {
    if (diag) pauli_group_kernel<double, true><<<nblocks, RB, 0, s>>>((const double2*)amps, len, g, partials);
    else pauli_group_kernel<double, false><<<nblocks, RB, 0, s>>>((const double2*)amps, len, g, partials);
  } else {
    if (diag) pauli_group_kernel<float, true><<<nblocks, RB, 0, s>>>((const float2*)amps, len, g, partials);
    else pauli_group_kernel<float, false><<<nblocks, RB, 0, s>>>((const float2*)amps, len, g, partials);
  }
  finish_kernel<NV><<<1, 32, 0, s>>>(partials, nblocks, out);
  return cudaGetLastError();
}

// ---- marginal probabilities ------------------------------------------------------
// k <= 10: per-block shared-memory histograms, summed by a second kernel.
template <typename Real>
__global__ void __launch_bounds__(RB) hist_kernel(const V2<Real>* __restrict__ amps, uint64_t len,
                                                  const uint32_t* __restrict__ qubits, uint32_t k,
                                                  double* __restrict__ partials) {
  extern __shared__ double hist[];
  const uint32_t dim = 1u << k;
  for (uint32_t i = threadIdx.x; i < dim; i += RB) hist[i] = 0.0;
  __shared__ uint32_t qs[16];
  if (threadIdx.x < k) qs[threadIdx.x] = qubits[threadIdx.x];
  __syncthreads();
  double v[2] = {0.0, 0.0};
  for (uint64_t i = (uint64_t)blockIdx.x * RB + threadIdx.x; i < len; i += (uint64_t)gridDim.x * RB) {
    const double p = abs2<Real>(ld_amp<Real>(amps + i));
    if (!isfinite(p)) {
      v[1] += 1.0;
      continue;
    }
    v[0] += p;
    uint32_t o = 0;
    for (uint32_t q = 0; q < k; ++q) o |= (uint32_t)((i >> qs[q]) & 1) << q;
    atomicAdd(&hist[o], p);
  }
  __syncthreads();
  double* out = partials + (size_t)blockIdx.x * (dim + 2);
  for (uint32_t i = threadIdx.x; i < dim; i += RB) out[2 + i] = hist[i];
  block_reduce_store<2>(v, out);
}

__global__ void hist_finish_kernel(const double* __restrict__ partials, uint32_t nblocks, uint32_t dim,
                                   double* __restrict__ out, double* __restrict__ norm_out) {
  for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < dim + 2; o += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t b = 0; b < nblocks; ++b) s += partials[(size_t)b * (dim + 2) + o];
    if (o < 2) norm_out[o] = s;
    else out[o - 2] = s;
  }
}

// k > 10: one thread per output entry sums its pre-images in index order.
template <typename Real>
__global__ void marginal_kernel(const V2<Real>* __restrict__ amps, uint32_t n, const uint32_t* __restrict__ qubits,
                                uint32_t k, double* __restrict__ out) {
  uint64_t qmask = 0;
  for (uint32_t q = 0; q < k; ++q) qmask |= 1ull << qubits[q];
  const uint64_t dim = 1ull << k, rest = 1ull << (n - k);
  for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < dim; o += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t fixed = 0;
    for (uint32_t q = 0; q < k; ++q) fixed |= ((o >> q) & 1) << qubits[q];
    double s = 0.0;
    for (uint64_t r = 0; r < rest; ++r) {
      // deposit r into the non-selected qubits
      uint64_t x = fixed, rr = r;
      for (uint32_t pos = 0; rr != 0 && pos < n; ++pos) {
        if ((qmask >> pos) & 1) continue;
        x |= (rr & 1) << pos;
        rr >>= 1;
      }
      s += abs2<Real>(ld_amp<Real>(amps + x));
    }
    out[o] = s;
  }
}

cudaError_t launch_probabilities(const void* amps, int precision, uint32_t n, const uint32_t* qubits_dev, uint32_t k,
                                 double* partials, uint32_t nblocks, double* out, double* norm_out, cudaStream_t s) {
  const uint64_t len = 1ull << n;
  if (k <= 10) {
    const uint32_t dim = 1u << k;
    const size_t sh = sizeof(double) * dim;
    if (precision == ALEPH_B200_F64)
      hist_kernel<double><<<nblocks, RB, sh, s>>>((const double2*)amps, len, qubits_dev, k, partials);
    else
      hist_kernel<float><<<nblocks, RB, sh, s>>>((const float2*)amps, len, qubits_dev, k, partials);
    hist_finish_kernel<<<(dim + 2 + 255) / 256, 256, 0, s>>>(partials, nblocks, dim, out, norm_out);
  } else {
    launch_norm(amps, precision, n, partials, nblocks, norm_out, s);
    const uint64_t dim = 1ull << k;
    const uint64_t b = (dim + 255) / 256;
    const unsigned blocks = (unsigned)(b > 148ull * 16 ? 148ull * 16 : b);
    if (precision == ALEPH_B200_F64)
      marginal_kernel<double><<<blocks, 256, 0, s>>>((const double2*)amps, n, qubits_dev, k, out);
    else
      marginal_kernel<float><<<blocks, 256, 0, s>>>((const float2*)amps, n, qubits_dev, k, out);
  }
  return cudaGetLastError();
}

}  // namespace ab
