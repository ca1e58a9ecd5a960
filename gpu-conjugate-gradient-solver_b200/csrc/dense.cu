// Dense inverse of an SPD matrix on the GPU, for coarsest levels too large
// for the host Cholesky (thousands of rows): in-place Gauss-Jordan
// elimination in FP64 without pivoting. For an SPD matrix the k-th pivot is
// the first diagonal entry of the k-th Schur complement, which is positive,
// so no pivoting is needed; a non-positive pivot means the matrix is not SPD.
//
// Step k (p = a_kk):
//     a_kk <- 1 / p
//     a_kj <- a_kj / p                       (j != k)
//     a_ij <- a_ij - a_ik a_kj / p           (i != k, j != k)
//     a_ik <- -a_ik / p                      (i != k)
// The pivot kernel saves column k and the scaled row k, so that the update
// kernel writes each entry once from values that no thread of it changes.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "dense.h"
#include "solver.h"

namespace gsb {

namespace {

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void gj_pivot_kernel(const double *__restrict__ a, int n, int k, double *__restrict__ colk,
                                double *__restrict__ rowk, int *__restrict__ bad) {
  const double p = a[static_cast<size_t>(k) * n + k];
  if (blockIdx.x == 0 && threadIdx.x == 0 && !(p > 0.0)) *bad = 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    colk[i] = a[static_cast<size_t>(i) * n + k];
    rowk[i] = a[static_cast<size_t>(k) * n + i] / p;
  }
}

__global__ void gj_update_kernel(double *__restrict__ a, int n, int k, const double *__restrict__ colk,
                                 const double *__restrict__ rowk) {
  const double p = colk[k];
  const size_t total = static_cast<size_t>(n) * n;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e / n), j = static_cast<int>(e % n);
    double v;
    if (i == k) v = j == k ? 1.0 / p : rowk[j];
    else if (j == k) v = -colk[i] / p;
    else v = fma(-colk[i], rowk[j], a[e]);
    a[e] = v;
  }
}

}  // namespace

void spd_inverse_device(const Csr &m, double *d_out, cudaStream_t s) {
  const int n = m.rows;
  if (m.cols != n) throw std::runtime_error("dense inverse: matrix must be square");
  if (n == 0) return;
  std::vector<double> h(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int e = m.rp[i]; e < m.rp[i + 1]; ++e) h[static_cast<size_t>(i) * n + m.ci[e]] += m.v[e];
  check(cudaMemcpyAsync(d_out, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, s), "dense upload");
  double *colk = nullptr, *rowk = nullptr;
  int *bad = nullptr;
  check(cudaMalloc(&colk, sizeof(double) * n), "dense scratch");
  check(cudaMalloc(&rowk, sizeof(double) * n), "dense scratch");
  check(cudaMalloc(&bad, sizeof(int)), "dense scratch");
  int hbad = 0;
  try {
    check(cudaMemsetAsync(bad, 0, sizeof(int), s), "dense flag");
    const int pb = std::min((n + 255) / 256, 1024);
    const size_t total = static_cast<size_t>(n) * n;
    const int ub = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
    for (int k = 0; k < n; ++k) {
      gj_pivot_kernel<<<pb, 256, 0, s>>>(d_out, n, k, colk, rowk, bad);
      gj_update_kernel<<<ub, 256, 0, s>>>(d_out, n, k, colk, rowk);
    }
    check(cudaGetLastError(), "dense inverse");
    check(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s), "dense flag");
    check(cudaStreamSynchronize(s), "dense inverse");
  } catch (...) {
    cudaFree(colk);
    cudaFree(rowk);
    cudaFree(bad);
    throw;
  }
  cudaFree(colk);
  cudaFree(rowk);
  cudaFree(bad);
  if (hbad) throw std::runtime_error("coarsest level matrix is not SPD (non-positive pivot)");
}

}  // namespace gsb

namespace gsb {

int dense_depth(const std::vector<int> &level_rows, int coarse_rows) {
  const int L = static_cast<int>(level_rows.size());
  if (coarse_rows <= 0) return L;
  for (int k = 1; k < L; ++k)
    if (level_rows[k] <= coarse_rows) return k + 1;
  return L;
}

}  // namespace gsb
