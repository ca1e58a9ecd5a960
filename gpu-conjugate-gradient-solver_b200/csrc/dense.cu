// Dense inverse of an SPD matrix on the GPU, for coarsest levels too large
// for the host Cholesky (thousands to tens of thousands of rows): the CSR
// matrix is scattered into a dense n x n array on the device, factorised
// A = L L^T and inverted from the factor by cuSOLVER (potrf + potri, FP64),
// and the lower triangle of the inverse is mirrored into the upper one. This is setup work; the per-solve
// dense matvec is the library's own kernel.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
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

void check_solver(cusolverStatus_t e, const char *what) {
  if (e != CUSOLVER_STATUS_SUCCESS) throw CudaError(std::string(what) + ": cuSOLVER status " + std::to_string(int(e)));
}

// a[i * n + ci[k]] += v[k] for the entries of row i (a zeroed before).
__global__ void csr_scatter_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                   const double *__restrict__ v, double *__restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) a[static_cast<size_t>(i) * n + ci[k]] += v[k];
}

// Row-major view: potri leaves the inverse in the column-major lower
// triangle, i.e. the row-major upper triangle (j >= i); copy it down.
__global__ void mirror_upper_kernel(int n, double *__restrict__ a) {
  const size_t total = static_cast<size_t>(n) * n;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e / n), j = static_cast<int>(e % n);
    if (j < i) a[e] = a[static_cast<size_t>(j) * n + i];
  }
}

template <typename T>
struct DevArray {
  T *p = nullptr;
  explicit DevArray(size_t n) { check(cudaMalloc(&p, sizeof(T) * (n == 0 ? 1 : n)), "dense scratch"); }
  ~DevArray() { cudaFree(p); }
  DevArray(const DevArray &) = delete;
  DevArray &operator=(const DevArray &) = delete;
};

}  // namespace

void spd_inverse_device(const Csr &m, double *d_out, cudaStream_t s) {
  const int n = m.rows;
  if (m.cols != n) throw std::runtime_error("dense inverse: matrix must be square");
  if (n == 0) return;
  const size_t total = static_cast<size_t>(n) * n;
  DevArray<int> rp(m.rp.size()), ci(m.ci.size());
  DevArray<double> v(m.v.size());
  check(cudaMemcpyAsync(rp.p, m.rp.data(), sizeof(int) * m.rp.size(), cudaMemcpyHostToDevice, s), "dense upload");
  if (!m.ci.empty()) {
    check(cudaMemcpyAsync(ci.p, m.ci.data(), sizeof(int) * m.ci.size(), cudaMemcpyHostToDevice, s), "dense upload");
    check(cudaMemcpyAsync(v.p, m.v.data(), sizeof(double) * m.v.size(), cudaMemcpyHostToDevice, s), "dense upload");
  }
  check(cudaMemsetAsync(d_out, 0, sizeof(double) * total, s), "dense zero");
  csr_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, rp.p, ci.p, v.p, d_out);
  check(cudaGetLastError(), "dense scatter");
  cusolverDnHandle_t h = nullptr;
  check_solver(cusolverDnCreate(&h), "cusolverDnCreate");
  int hinfo[2] = {0, 0};
  try {
    check_solver(cusolverDnSetStream(h, s), "cusolverDnSetStream");
    int lw_f = 0, lw_i = 0;
    check_solver(cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, d_out, n, &lw_f), "potrf workspace");
    check_solver(cusolverDnDpotri_bufferSize(h, CUBLAS_FILL_MODE_LOWER, n, d_out, n, &lw_i), "potri workspace");
    DevArray<double> work(static_cast<size_t>(std::max(lw_f, lw_i)));
    DevArray<int> info(2);
    check(cudaMemsetAsync(info.p, 0, 2 * sizeof(int), s), "dense info");
    // the matrix is symmetric, so its row-major array is also its
    // column-major array: factorise its lower triangle
    check_solver(cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, n, d_out, n, work.p, lw_f, info.p), "potrf");
    check(cudaMemcpyAsync(&hinfo[0], info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "dense info");
    check(cudaStreamSynchronize(s), "potrf");
    if (hinfo[0] == 0) {
      check_solver(cusolverDnDpotri(h, CUBLAS_FILL_MODE_LOWER, n, d_out, n, work.p, lw_i, info.p + 1), "potri");
      check(cudaMemcpyAsync(&hinfo[1], info.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s), "dense info");
      const int grid = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
      mirror_upper_kernel<<<grid, 256, 0, s>>>(n, d_out);
      check(cudaGetLastError(), "dense mirror");
      check(cudaStreamSynchronize(s), "potri");
    }
  } catch (...) {
    cusolverDnDestroy(h);
    throw;
  }
  cusolverDnDestroy(h);
  if (hinfo[0] != 0 || hinfo[1] != 0)
    throw std::runtime_error("coarsest level matrix is not SPD (Cholesky failed)");
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
