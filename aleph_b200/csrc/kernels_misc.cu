// kernels_misc.cu — shared-memory whole-state pass (n <= 12), dense k-qubit
// UnitaryKq pass, state initialisation, precision conversion and the bit
// permutation of unpermute_state.
//
// Semantics follow the reference kernels: pair/quartet butterflies
// (crates/aleph-sv/src/kernels/aos.rs:192-223, :1335-1394), MSB-first operand
// order (crates/aleph-sv/src/kernels/unitary_kq.rs:66-96), controls as an AND
// mask over the basis index (aos.rs:198-205).

#include <cstdio>

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

// ---- renormalisation (end of a tensor-core gate stream) ----------------------
// Tensor-core FP32 accumulation drifts the state norm systematically (by
// ~1e-6 per block pass); one FP64 norm reduction and one rescale pass restore
// |psi| = 1 without a host round trip.
template <typename Real>
__global__ void rescale_kernel(V2<Real>* __restrict__ amps, uint64_t len, const double* __restrict__ norm2) {
  const double s = norm2[0] > 0.0 ? rsqrt(norm2[0]) : 1.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
    const V2<Real> a = ld_amp<Real>(amps + i);
    st_amp<Real>(amps + i, mk<Real>((Real)(a.x * s), (Real)(a.y * s)));
  }
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
