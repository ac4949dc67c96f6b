// kernels_peak.cu — the FP64 issue rate of this device's CUDA cores, measured.
//
// The plain FP64 tile passes are bound by double-precision FMA issue, not by
// HBM, once several gates fuse into a pass. Their roofline needs the DFMA
// rate the SMs actually sustain at the clock they run at, which no copy or
// GEMM benchmark gives. This kernel runs 8 independent FMA chains per thread
// (enough to cover the FMA latency) over a full-occupancy grid and nothing
// else: no memory traffic but one store per thread at the end.

#include "common.cuh"

namespace ab {

constexpr int PEAK_CHAINS = 8;

__global__ void __launch_bounds__(256) dfma_peak_kernel(double* out, uint32_t iters, double a, double b) {
  double x[PEAK_CHAINS];
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) s += x[c];
  out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

// DFMA per launch: blocks * 256 * iters * 16 * PEAK_CHAINS.
cudaError_t launch_dfma_peak(double* out, uint32_t blocks, uint32_t iters, cudaStream_t s) {
  // a slightly below 1 and b small keep the values finite and normal
  dfma_peak_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.999999, 1e-7);
  return cudaGetLastError();
}

double dfma_per_launch(uint32_t blocks, uint32_t iters) {
  return (double)blocks * 256.0 * iters * 16.0 * PEAK_CHAINS;
}

}  // namespace ab
