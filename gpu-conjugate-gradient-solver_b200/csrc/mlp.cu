// Learned relaxation weights: a small MLP, trained and evaluated with these
// hand-written kernels (FP32).
//
//   features (8) -> 32, tanh -> 32, tanh -> 1 -> omega = 2 sigmoid(z),
//   clamped to [0.02, 1.98] (zero gradient outside) so that omega stays
//   strictly inside (0, 2) even where the sigmoid saturates
//
// One sample per (level, colour) of a hierarchy; the predicted omega weights
// that colour's Gauss-Seidel updates in both the forward and the backward
// sweep (pre- and post-smoothing alike), which keeps the V-cycle symmetric
// positive definite. Parameters, flat FP32: W1[32][8], b1[32], W2[32][32],
// b2[32], W3[32], b3 (1377 values).
//
// All buffers are the caller's: the forward pass stores per-sample
// activations in `cache` (65 floats per sample), the backward pass its
// per-sample deltas in `delta` (65 floats per sample) and the parameter
// gradient in `grad` (1377 floats), summed over samples in sample order by
// one thread per parameter (deterministic).
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "mlp.h"
#include "solver.h"

namespace gsb {

namespace {

constexpr int kIn = kMlpIn, kH = kMlpHidden;
constexpr int oW1 = 0, oB1 = kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
constexpr int kCache = 2 * kH + 1;  // h1, h2, z
constexpr float kOmegaMin = 0.02f, kOmegaMax = 1.98f;

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void mlp_forward_kernel(const float *__restrict__ p, const float *__restrict__ f, int n,
                                   float *__restrict__ omega, float *__restrict__ cache) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[kIn], h1[kH], h2[kH];
  for (int j = 0; j < kIn; ++j) x[j] = f[s * kIn + j];
  for (int i = 0; i < kH; ++i) {
    float a = p[oB1 + i];
    for (int j = 0; j < kIn; ++j) a = fmaf(p[oW1 + i * kIn + j], x[j], a);
    h1[i] = tanhf(a);
  }
  for (int i = 0; i < kH; ++i) {
    float a = p[oB2 + i];
    for (int j = 0; j < kH; ++j) a = fmaf(p[oW2 + i * kH + j], h1[j], a);
    h2[i] = tanhf(a);
  }
  float z = p[oB3];
  for (int j = 0; j < kH; ++j) z = fmaf(p[oW3 + j], h2[j], z);
  omega[s] = fminf(fmaxf(2.0f / (1.0f + expf(-z)), kOmegaMin), kOmegaMax);
  if (cache != nullptr) {
    float *c = cache + static_cast<size_t>(s) * kCache;
    for (int i = 0; i < kH; ++i) c[i] = h1[i], c[kH + i] = h2[i];
    c[2 * kH] = z;
  }
}

// Per-sample deltas from the upstream gradient g = dL/domega.
__global__ void mlp_delta_kernel(const float *__restrict__ p, int n, const float *__restrict__ cache,
                                 const float *__restrict__ g, float *__restrict__ delta) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float *c = cache + static_cast<size_t>(s) * kCache;
  float *d = delta + static_cast<size_t>(s) * kCache;
  const float z = c[2 * kH];
  const float sg = 1.0f / (1.0f + expf(-z));
  const float w = 2.0f * sg;
  const float dz = (w < kOmegaMin || w > kOmegaMax) ? 0.0f : g[s] * 2.0f * sg * (1.0f - sg);
  float d2[kH];
  for (int i = 0; i < kH; ++i) {
    const float h = c[kH + i];
    d2[i] = dz * p[oW3 + i] * (1.0f - h * h);
  }
  for (int j = 0; j < kH; ++j) {
    float a = 0.0f;
    for (int i = 0; i < kH; ++i) a = fmaf(p[oW2 + i * kH + j], d2[i], a);
    const float h = c[j];
    d[j] = a * (1.0f - h * h);  // delta of layer 1
  }
  for (int i = 0; i < kH; ++i) d[kH + i] = d2[i];
  d[2 * kH] = dz;
}

// One thread per parameter, samples summed in order.
__global__ void mlp_grad_kernel(const float *__restrict__ f, int n, const float *__restrict__ cache,
                                const float *__restrict__ delta, float *__restrict__ grad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kMlpParams) return;
  float acc = 0.0f;
  for (int s = 0; s < n; ++s) {
    const float *c = cache + static_cast<size_t>(s) * kCache;
    const float *d = delta + static_cast<size_t>(s) * kCache;
    float v;
    if (q < oB1) v = d[q / kIn] * f[s * kIn + q % kIn];
    else if (q < oW2) v = d[q - oB1];
    else if (q < oB2) v = d[kH + (q - oW2) / kH] * c[(q - oW2) % kH];
    else if (q < oW3) v = d[kH + (q - oB2)];
    else if (q < oB3) v = d[2 * kH] * c[kH + (q - oW3)];
    else v = d[2 * kH];
    acc += v;
  }
  grad[q] = acc;
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int np, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.0f - b1) * gq;
  const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

}  // namespace

void mlp_forward(const float *params, const float *feats, int n, float *omega, float *cache,
                 cudaStream_t s) {
  if (n <= 0) return;
  mlp_forward_kernel<<<(n + 127) / 128, 128, 0, s>>>(params, feats, n, omega, cache);
  check(cudaGetLastError(), "mlp forward");
}

void mlp_backward(const float *params, const float *feats, int n, const float *cache,
                  const float *upstream, float *delta, float *grad, cudaStream_t s) {
  if (n <= 0) return;
  mlp_delta_kernel<<<(n + 127) / 128, 128, 0, s>>>(params, n, cache, upstream, delta);
  mlp_grad_kernel<<<(kMlpParams + 127) / 128, 128, 0, s>>>(feats, n, cache, delta, grad);
  check(cudaGetLastError(), "mlp backward");
}

void mlp_adam(float *params, const float *grad, float *m, float *v, int np, float lr, float b1,
              float b2, float eps, int step, cudaStream_t s) {
  if (step < 1) throw std::runtime_error("adam step counts from 1");
  const float c1 = 1.0f - powf(b1, static_cast<float>(step));
  const float c2 = 1.0f - powf(b2, static_cast<float>(step));
  adam_kernel<<<(np + 255) / 256, 256, 0, s>>>(params, grad, m, v, np, lr, b1, b2, eps, c1, c2);
  check(cudaGetLastError(), "adam");
}

}  // namespace gsb
