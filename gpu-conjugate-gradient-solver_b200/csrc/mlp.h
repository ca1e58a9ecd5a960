// Learned relaxation weights: MLP kernels (see mlp.cu).
#pragma once

#include <cuda_runtime.h>

namespace gsb {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 32;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1;
constexpr int kMlpCache = 2 * kMlpHidden + 1;

void mlp_forward(const float *params, const float *feats, int n, float *omega, float *cache, cudaStream_t s);
void mlp_backward(const float *params, const float *feats, int n, const float *cache, const float *upstream,
                  float *delta, float *grad, cudaStream_t s);
void mlp_adam(float *params, const float *grad, float *m, float *v, int np, float lr, float b1, float b2,
              float eps, int step, cudaStream_t s);

}  // namespace gsb
