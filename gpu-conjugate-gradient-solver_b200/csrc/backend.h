// Kernel-level operations of the reference's Backend (see backend.cu).
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "gpusolver_b200.h"
#include "solver.h"

namespace gsb {

// A CSR matrix on the device in the caller's row order
// (CudaDeviceCSRMatrix, src/cuda/CudaDeviceCSRMatrix.cc:28-116).
struct DeviceCsr {
  int rows = 0, cols = 0, nnz = 0, dtype = GS_F64;
  int *rp = nullptr, *ci = nullptr;
  void *v = nullptr;
  bool diag_ok = false;  // square with every diagonal entry present and nonzero
  ~DeviceCsr();
};

DeviceCsr *device_csr_create(int rows, int cols, const int *rp, const int *ci, const void *val, int dtype);
void device_csr_update_values(DeviceCsr *m, const void *val, long long count);
void spmv(const DeviceCsr *m, const void *x, void *y, cudaStream_t s);
void gauss_seidel_color(const DeviceCsr *m, const int *order, long long start, long long count,
                        const void *rhs, void *x, double omega, cudaStream_t s);
void block_gauss_seidel_color3x3(const DeviceCsr *m, const int *order, long long start, long long count,
                                 const void *dinv, const void *rhs, void *x, double omega, cudaStream_t s);
void apply_block_inverses3x3(long long n, const void *dinv, const void *r, void *c, int dtype, cudaStream_t s);
void dot(long long n, const void *x, const void *y, void *result, int dtype, cudaStream_t s);
// dot with caller-provided scratch (kDotBlocks partials + a zeroed ticket)
void launch_dot(long long n, const void *x, const void *y, void *result, int dtype, double *partials,
                unsigned int *ticket, cudaStream_t s);
// dot with its scratch in a fixed device array of the library (no allocation)
void dot_noalloc(long long n, const void *x, const void *y, void *result, int dtype, cudaStream_t s);
void vector_op(int op, long long n, const void *x, void *y, double alpha, const void *alpha_dev,
               int dtype, cudaStream_t s);
void scalar_op(int op, const void *a, const void *b, void *out, double value, int dtype, cudaStream_t s);

}  // namespace gsb
