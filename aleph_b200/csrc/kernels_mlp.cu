// kernels_mlp.cu — the learned fusion planner's cost model: a small FP32
// MLP (F inputs -> 3 hidden layers of H ReLU units -> 1 output) that predicts
// a pass's device time from its features, trained on the per-pass timings
// the engine records. Forward, backward (MSE loss) and Adam run in these
// kernels; shapes are small (H = 128), so each layer is one SIMT kernel with
// one thread per output element and the weights read through L1.
//
// Parameter layout (one flat FP32 buffer): for layer l = 0..3 with
// (in, out) = (F, H), (H, H), (H, H), (H, 1): W_l[out][in] row-major, then b_l[out].

#include "common.cuh"

namespace ab {

namespace mlp {

constexpr int BS = 256;

// Y[b][o] = act(sum_i X[b][i] W[o][i] + bias[o]); act = ReLU when relu != 0.
__global__ void fwd_kernel(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ bias,
                           float* __restrict__ Y, int B, int I, int O, int relu) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * O) return;
  const int b = idx / O, o = idx % O;
  const float* x = X + (size_t)b * I;
  const float* w = W + (size_t)o * I;
  float s = bias[o];
  for (int i = 0; i < I; ++i) s = fmaf(x[i], w[i], s);
  Y[idx] = relu && s < 0.f ? 0.f : s;
}

// dZ = dY * (Y > 0) in place (ReLU derivative through the layer output Y).
__global__ void relu_bwd_kernel(float* __restrict__ dY, const float* __restrict__ Y, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < n && Y[idx] <= 0.f) dY[idx] = 0.f;
}

// dX[b][i] = sum_o dZ[b][o] W[o][i]
__global__ void bwd_data_kernel(const float* __restrict__ dZ, const float* __restrict__ W, float* __restrict__ dX,
                                int B, int I, int O) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= B * I) return;
  const int b = idx / I, i = idx % I;
  const float* dz = dZ + (size_t)b * O;
  float s = 0.f;
  for (int o = 0; o < O; ++o) s = fmaf(dz[o], W[(size_t)o * I + i], s);
  dX[idx] = s;
}

// dW[o][i] = sum_b dZ[b][o] X[b][i]; db[o] = sum_b dZ[b][o] (one thread per weight; i == I: the bias)
__global__ void bwd_weight_kernel(const float* __restrict__ dZ, const float* __restrict__ X, float* __restrict__ dW,
                                  float* __restrict__ db, int B, int I, int O) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= O * (I + 1)) return;
  const int o = idx / (I + 1), i = idx % (I + 1);
  float s = 0.f;
  if (i < I) {
    for (int b = 0; b < B; ++b) s = fmaf(dZ[(size_t)b * O + o], X[(size_t)b * I + i], s);
    dW[(size_t)o * I + i] = s;
  } else {
    for (int b = 0; b < B; ++b) s += dZ[(size_t)b * O + o];
    db[o] = s;
  }
}

// MSE: loss = mean((yhat - y)^2), dyhat = 2 (yhat - y) / B; loss accumulated by one block.
__global__ void mse_kernel(const float* __restrict__ yhat, const float* __restrict__ y, float* __restrict__ dy,
                           float* __restrict__ loss, int B) {
  __shared__ float part[BS];
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const float d = yhat[b] - y[b];
    dy[b] = 2.f * d / (float)B;
    s += d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k; k >>= 1) {
    if (threadIdx.x < k) part[threadIdx.x] += part[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = part[0] / (float)B;
}

// Adam (Kingma & Ba 2015) with bias correction; t is the 1-based step.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const float gi = g[idx];
  const float mi = b1 * m[idx] + (1.f - b1) * gi;
  const float vi = b2 * v[idx] + (1.f - b2) * gi * gi;
  m[idx] = mi;
  v[idx] = vi;
  p[idx] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline unsigned blocks(long long n) { return (unsigned)((n + BS - 1) / BS); }

}  // namespace mlp

size_t mlp_param_count(int F, int H) {
  return (size_t)H * F + H + 2 * ((size_t)H * H + H) + H + 1;
}

// Layer l's (in, out) and its parameter offsets.
static void layer_shape(int l, int F, int H, int* in, int* out, size_t* w_off, size_t* b_off) {
  const int ins[4] = {F, H, H, H}, outs[4] = {H, H, H, 1};
  size_t off = 0;
  for (int k = 0; k < l; ++k) off += (size_t)ins[k] * outs[k] + outs[k];
  *in = ins[l];
  *out = outs[l];
  *w_off = off;
  *b_off = off + (size_t)ins[l] * outs[l];
}

// acts: 4 layer outputs of B x {H, H, H, 1}, laid out back to back.
cudaError_t mlp_forward(const float* params, const float* X, float* acts, int B, int F, int H, cudaStream_t s) {
  const float* in = X;
  size_t a_off = 0;
  for (int l = 0; l < 4; ++l) {
    int I, O;
    size_t wo, bo;
    layer_shape(l, F, H, &I, &O, &wo, &bo);
    float* out = acts + a_off;
    mlp::fwd_kernel<<<mlp::blocks((long long)B * O), mlp::BS, 0, s>>>(in, params + wo, params + bo, out, B, I, O,
                                                                      l < 3 ? 1 : 0);
    in = out;
    a_off += (size_t)B * O;
  }
  return cudaGetLastError();
}

// Gradients of the MSE loss into grads (same layout as params); dbuf holds
// 2 x B x H floats of scratch; loss_dev receives the loss.
cudaError_t mlp_backward(const float* params, const float* X, const float* acts, const float* y, float* grads,
                         float* dbuf, float* loss_dev, int B, int F, int H, cudaStream_t s) {
  const float* yhat = acts + (size_t)3 * B * H;
  float* dcur = dbuf;               // gradient w.r.t. the current layer's output
  float* dnext = dbuf + (size_t)B * H;
  mlp::mse_kernel<<<1, mlp::BS, 0, s>>>(yhat, y, dcur, loss_dev, B);
  for (int l = 3; l >= 0; --l) {
    int I, O;
    size_t wo, bo;
    layer_shape(l, F, H, &I, &O, &wo, &bo);
    const float* Y = acts + (size_t)l * B * H;  // this layer's output (layer 3: B x 1)
    const float* Xin = l == 0 ? X : acts + (size_t)(l - 1) * B * H;
    if (l < 3) mlp::relu_bwd_kernel<<<mlp::blocks((long long)B * O), mlp::BS, 0, s>>>(dcur, Y, B * O);
    mlp::bwd_weight_kernel<<<mlp::blocks((long long)O * (I + 1)), mlp::BS, 0, s>>>(dcur, Xin, grads + wo,
                                                                                    grads + bo, B, I, O);
    if (l > 0) {
      mlp::bwd_data_kernel<<<mlp::blocks((long long)B * I), mlp::BS, 0, s>>>(dcur, params + wo, dnext, B, I, O);
      float* t = dcur;
      dcur = dnext;
      dnext = t;
    }
  }
  return cudaGetLastError();
}

cudaError_t mlp_adam(float* params, const float* grads, float* m, float* v, size_t n, float lr, int step,
                     cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  mlp::adam_kernel<<<mlp::blocks((long long)n), mlp::BS, 0, s>>>(params, grads, m, v, (int)n, lr, b1, b2, 1e-8f, c1,
                                                                 c2);
  return cudaGetLastError();
}

}  // namespace ab
