// Kernel-level entry points: the reference's Backend operations
// (include/GPUSolver/Backend.h:47-114) on device pointers, FP32 or FP64.
// The AMG-PCG solver does not go through these (it runs fused kernels on
// its own layouts); they exist so code written against the reference's
// Backend can call single operations, with the reference's semantics:
//   encodeSpmv                    y = A x                     (CSR, any row order)
//   encodeGaussSeidelColor        one colour pass through an index list
//   encodeBlockGaussSeidelColor3x3  (colorStart, colorCount) reading
//   encodeApplyBlockInverses3x3   c_b = D_b^-1 r_b
//   encodeDot                     deterministic two-stage reduction
//   encodeAxpy/Scale/Copy/SetZero/ScaleVector, scalar divide/multiply/...
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "backend.h"
#include "kernels.cuh"

namespace gsb {

namespace {

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kDotBlocks = 296;  // 2 blocks per SM of a 148-SM B200

// Per-device scratch of the reduction entry points: partial sums of each
// block and the arrival ticket of the last-block-done pattern. Allocated
// once per device on first use and kept until exit.
struct DotScratch {
  double *partials = nullptr;  // kDotBlocks
  unsigned int *ticket = nullptr;
};

DotScratch &dot_scratch() {
  static std::mutex mu;
  static std::vector<DotScratch> per_device;
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (static_cast<int>(per_device.size()) <= dev) per_device.resize(dev + 1);
  DotScratch &s = per_device[dev];
  if (s.partials == nullptr) {
    check(cudaMalloc(&s.partials, sizeof(double) * kDotBlocks), "dot scratch");
    check(cudaMalloc(&s.ticket, sizeof(unsigned int)), "dot ticket");
    check(cudaMemset(s.ticket, 0, sizeof(unsigned int)), "dot ticket clear");
  }
  return s;
}

// result = x . y, sequential-order partials per block, the last block adds
// the partials in block order (deterministic for a given n).
template <typename T>
__global__ void __launch_bounds__(256) dot_kernel(int n, const T *__restrict__ x,
                                                  const T *__restrict__ y, T *result,
                                                  double *partials, unsigned int *ticket) {
  __shared__ double smem[32];
  double acc[1] = {0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    acc[0] = fma(double(x[i]), double(y[i]), acc[0]);
  if (grid_sum<1>(acc, partials, ticket, smem) && threadIdx.x == 0) *result = T(acc[0]);
}

template <typename T>
__global__ void gs_color_indirect_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                         const T *__restrict__ v, const int *__restrict__ order,
                                         long long start, long long count, const T *__restrict__ rhs,
                                         T *__restrict__ x, T omega) {
  // 8 lanes per listed row
  const int sub = threadIdx.x & 7;
  const long long i = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 3;
  const bool valid = i < count;
  const int row = valid ? order[start + i] : 0;
  T off = T(0), diag = T(0);
  if (valid)
    for (int k = rp[row] + sub; k < rp[row + 1]; k += 8) {
      const int c = ci[k];
      if (c == row) diag = v[k];
      else off = fma(v[k], x[c], off);
    }
  for (int o = 4; o > 0; o >>= 1) {
    off += __shfl_xor_sync(0xffffffffu, off, o, 8);
    diag += __shfl_xor_sync(0xffffffffu, diag, o, 8);
  }
  if (valid && sub == 0) x[row] = (T(1) - omega) * x[row] + omega * ((rhs[row] - off) / diag);
}

template <typename T>
__global__ void block_gs_indirect_kernel(const int *__restrict__ rp, const int *__restrict__ ci,
                                         const T *__restrict__ v, const int *__restrict__ order,
                                         long long start, long long count,
                                         const T *__restrict__ dinv, const T *__restrict__ rhs,
                                         T *__restrict__ x, T omega) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int blk = order[start + i], r0 = 3 * blk;
  T res[3];
  for (int l = 0; l < 3; ++l) {
    T s = T(0);
    for (int k = rp[r0 + l]; k < rp[r0 + l + 1]; ++k) {
      const int c = ci[k];
      if (c >= r0 && c < r0 + 3) continue;
      s = fma(v[k], x[c], s);
    }
    res[l] = rhs[r0 + l] - s;
  }
  const T *bi = dinv + 9 * static_cast<size_t>(blk);
  for (int l = 0; l < 3; ++l) {
    T nv = bi[3 * l] * res[0];
    nv = fma(bi[3 * l + 1], res[1], nv);
    nv = fma(bi[3 * l + 2], res[2], nv);
    x[r0 + l] = (T(1) - omega) * x[r0 + l] + omega * nv;
  }
}

template <typename T>
__global__ void block_inverse_apply_kernel(long long nblocks, const T *__restrict__ dinv,
                                           const T *__restrict__ r, T *__restrict__ c) {
  const long long b = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const T *bi = dinv + 9 * b;
  const T r0 = r[3 * b], r1 = r[3 * b + 1], r2 = r[3 * b + 2];
  for (int l = 0; l < 3; ++l) c[3 * b + l] = fma(bi[3 * l], r0, fma(bi[3 * l + 1], r1, bi[3 * l + 2] * r2));
}

// y op= alpha x, alpha from the host (alpha_dev == nullptr) or the device
template <typename T>
__global__ void vec_kernel(int op, long long n, const T *__restrict__ x, T *__restrict__ y, T alpha,
                           const T *alpha_dev) {
  const T a = alpha_dev != nullptr ? *alpha_dev : alpha;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    switch (op) {
      case GS_VEC_AXPY: y[i] = fma(a, x[i], y[i]); break;
      case GS_VEC_SCALE: y[i] = a * y[i]; break;
      case GS_VEC_COPY: y[i] = x[i]; break;
      case GS_VEC_SET_ZERO: y[i] = T(0); break;
      case GS_VEC_SCALE_BY_VECTOR: y[i] = x[i] * y[i]; break;
      default: break;
    }
  }
}

template <typename T>
__global__ void scalar_kernel(int op, const T *a, const T *b, T *out, T value) {
  switch (op) {
    case GS_SCALAR_DIVIDE: *out = *a / *b; break;
    case GS_SCALAR_MULTIPLY: *out = *a * *b; break;
    case GS_SCALAR_SET: *out = value; break;
    case GS_SCALAR_COPY: *out = *a; break;
    case GS_SCALAR_NEGATE: *out = -*a; break;
    case GS_SCALAR_SQRT: *out = sqrt(*a); break;
    default: break;
  }
}

inline int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return static_cast<int>(b);
}

}  // namespace

DeviceCsr::~DeviceCsr() {
  cudaFree(rp);
  cudaFree(ci);
  cudaFree(v);
}

DeviceCsr *device_csr_create(int rows, int cols, const int *rp, const int *ci, const void *val,
                             int dtype) {
  if (rows <= 0 || cols <= 0) throw std::runtime_error("DeviceCSRMatrix: matrix dimensions must be nonzero.");
  if (dtype != GS_F32 && dtype != GS_F64) throw std::runtime_error("dtype must be GS_F32 or GS_F64");
  std::unique_ptr<DeviceCsr> m(new DeviceCsr);
  m->rows = rows;
  m->cols = cols;
  m->nnz = rp[rows];
  m->dtype = dtype;
  const size_t vs = dtype == GS_F32 ? 4 : 8;
  check(cudaMalloc(&m->rp, sizeof(int) * (rows + 1)), "csr rows");
  check(cudaMalloc(&m->ci, sizeof(int) * (m->nnz > 0 ? m->nnz : 1)), "csr cols");
  check(cudaMalloc(&m->v, vs * (m->nnz > 0 ? m->nnz : 1)), "csr values");
  check(cudaMemcpy(m->rp, rp, sizeof(int) * (rows + 1), cudaMemcpyHostToDevice), "csr rows");
  if (m->nnz > 0) {
    check(cudaMemcpy(m->ci, ci, sizeof(int) * m->nnz, cudaMemcpyHostToDevice), "csr cols");
    check(cudaMemcpy(m->v, val, vs * m->nnz, cudaMemcpyHostToDevice), "csr values");
  }
  // zero or missing diagonal: the reference's CPU backend refuses to smooth
  // such a matrix (src/CPU/CPUBackend.cc:248-267)
  m->diag_ok = rows == cols;
  for (int r = 0; r < rows && m->diag_ok; ++r) {
    bool found = false;
    for (int k = rp[r]; k < rp[r + 1]; ++k)
      if (ci[k] == r) {
        const double d = dtype == GS_F32 ? double(static_cast<const float *>(val)[k])
                                         : static_cast<const double *>(val)[k];
        found = std::fabs(d) >= 1e-12;
      }
    m->diag_ok = found;
  }
  return m.release();
}

void device_csr_update_values(DeviceCsr *m, const void *val, long long count) {
  if (count != m->nnz) throw std::runtime_error("DeviceCSRMatrix::updateValues: size mismatch.");
  const size_t vs = m->dtype == GS_F32 ? 4 : 8;
  check(cudaMemcpy(m->v, val, vs * m->nnz, cudaMemcpyHostToDevice), "csr update");
}

void spmv(const DeviceCsr *m, const void *x, void *y, cudaStream_t s) {
  const int gb = std::min((m->rows * 8 + 255) / 256, 148 * 16);
  if (m->dtype == GS_F32) {
    CsrvView<float> v{m->rows, m->rp, m->ci, static_cast<const float *>(m->v), nullptr};
    csrv_spmv_kernel<float, float, kSpmvSet, 8><<<gb, 256, 0, s>>>(v, static_cast<const float *>(x), static_cast<float *>(y), nullptr, nullptr);
  } else {
    CsrvView<double> v{m->rows, m->rp, m->ci, static_cast<const double *>(m->v), nullptr};
    csrv_spmv_kernel<double, double, kSpmvSet, 8><<<gb, 256, 0, s>>>(v, static_cast<const double *>(x), static_cast<double *>(y), nullptr, nullptr);
  }
  check(cudaGetLastError(), "spmv");
}

void gauss_seidel_color(const DeviceCsr *m, const int *order, long long start, long long count,
                        const void *rhs, void *x, double omega, cudaStream_t s) {
  if (!m->diag_ok) throw std::runtime_error("encodeGaussSeidelColor: zero diagonal entry.");
  if (count <= 0) return;
  const int gb = static_cast<int>((count * 8 + 255) / 256);
  if (m->dtype == GS_F32)
    gs_color_indirect_kernel<float><<<gb, 256, 0, s>>>(m->rows, m->rp, m->ci, static_cast<const float *>(m->v), order, start, count, static_cast<const float *>(rhs), static_cast<float *>(x), float(omega));
  else
    gs_color_indirect_kernel<double><<<gb, 256, 0, s>>>(m->rows, m->rp, m->ci, static_cast<const double *>(m->v), order, start, count, static_cast<const double *>(rhs), static_cast<double *>(x), omega);
  check(cudaGetLastError(), "gauss-seidel colour");
}

void block_gauss_seidel_color3x3(const DeviceCsr *m, const int *order, long long start, long long count,
                                 const void *dinv, const void *rhs, void *x, double omega, cudaStream_t s) {
  if (m->rows % 3 != 0) throw std::runtime_error("3x3 block smoother requires number of DOFs divisible by 3.");
  if (count <= 0) return;
  const int gb = static_cast<int>((count + 255) / 256);
  if (m->dtype == GS_F32)
    block_gs_indirect_kernel<float><<<gb, 256, 0, s>>>(m->rp, m->ci, static_cast<const float *>(m->v), order, start, count, static_cast<const float *>(dinv), static_cast<const float *>(rhs), static_cast<float *>(x), float(omega));
  else
    block_gs_indirect_kernel<double><<<gb, 256, 0, s>>>(m->rp, m->ci, static_cast<const double *>(m->v), order, start, count, static_cast<const double *>(dinv), static_cast<const double *>(rhs), static_cast<double *>(x), omega);
  check(cudaGetLastError(), "block gauss-seidel colour");
}

void apply_block_inverses3x3(long long n, const void *dinv, const void *r, void *c, int dtype,
                             cudaStream_t s) {
  if (n % 3 != 0) throw std::runtime_error("encodeApplyBlockInverses3x3: size not divisible by 3");
  const long long nb = n / 3;
  if (nb == 0) return;
  const int gb = static_cast<int>((nb + 255) / 256);
  if (dtype == GS_F32)
    block_inverse_apply_kernel<float><<<gb, 256, 0, s>>>(nb, static_cast<const float *>(dinv), static_cast<const float *>(r), static_cast<float *>(c));
  else
    block_inverse_apply_kernel<double><<<gb, 256, 0, s>>>(nb, static_cast<const double *>(dinv), static_cast<const double *>(r), static_cast<double *>(c));
  check(cudaGetLastError(), "apply block inverses");
}

void launch_dot(long long n, const void *x, const void *y, void *result, int dtype, double *partials,
                unsigned int *ticket, cudaStream_t s) {
  if (n < 0 || n > 0x7fffffffLL) throw std::runtime_error("encodeDot: bad size");
  const int gb = std::min(grid_for(n), kDotBlocks);
  if (dtype == GS_F32)
    dot_kernel<float><<<gb, 256, 0, s>>>(static_cast<int>(n), static_cast<const float *>(x), static_cast<const float *>(y), static_cast<float *>(result), partials, ticket);
  else
    dot_kernel<double><<<gb, 256, 0, s>>>(static_cast<int>(n), static_cast<const double *>(x), static_cast<const double *>(y), static_cast<double *>(result), partials, ticket);
  check(cudaGetLastError(), "dot");
}

void dot(long long n, const void *x, const void *y, void *result, int dtype, cudaStream_t s) {
  DotScratch &sc = dot_scratch();
  launch_dot(n, x, y, result, dtype, sc.partials, sc.ticket, s);
}

// ---- dot product that allocates nothing ---------------------------------------
// Some callers cannot allocate device memory when they need a dot product:
// a simulation that reserves all of the GPU's memory for its own pool at
// start-up, or a time-critical loop that must not take cudaMalloc's implicit
// device synchronisation. For them, gs_dot_noalloc keeps the reduction's
// scratch (one partial sum per block and the last-block ticket) in the
// fixed array below, which is part of the library's device image: no call
// allocates anything from the caller's point of view. The array takes
// device memory on a GPU when the library's device image is loaded there.
// With CUDA's default lazy module loading that happens at the library's
// first GPU call on that device (any gs_* call that touches the GPU, this
// one included), which may itself need a little device memory: make that
// first call before the caller's pool claims the GPU's memory, or run with
// CUDA_MODULE_LOADING=EAGER. From then on each such GPU holds these
// 32 KB + 256 bytes until the process exits.
constexpr int kNoAllocPartials = 4096;              // partial sums, one per block
constexpr long long kNoAllocChunk = 2048;           // elements per block (256 threads x 8)
constexpr long long kNoAllocMaxN = kNoAllocPartials * kNoAllocChunk;  // 8,388,608 elements
static __device__ __align__(256) unsigned char g_dot_scratch[kNoAllocPartials * sizeof(double) + 256];

namespace {

// Device address of g_dot_scratch on the current device. In host code the
// name g_dot_scratch is only a host-side stand-in, so the address is looked
// up with cudaGetSymbolAddress with the device current. The lookup is made on
// every call (once the image is loaded it allocates nothing), so a context
// that was reset and re-created never sees a stale address.
unsigned char *noalloc_scratch_address() {
  void *ptr = nullptr;
  check(cudaGetSymbolAddress(&ptr, g_dot_scratch), "cudaGetSymbolAddress(g_dot_scratch)");
  return static_cast<unsigned char *>(ptr);
}

}  // namespace

void dot_noalloc(long long n, const void *x, const void *y, void *result, int dtype, cudaStream_t s) {
  if (n < 0) throw std::runtime_error("gs_dot_noalloc: negative size");
  if (n > kNoAllocMaxN)
    throw std::runtime_error("gs_dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                             std::to_string(kNoAllocMaxN) + " elements of its fixed scratch; use gs_dot");
  unsigned char *base = noalloc_scratch_address();
  double *partials = reinterpret_cast<double *>(base);
  unsigned int *ticket = reinterpret_cast<unsigned int *>(base + kNoAllocPartials * sizeof(double));
  // the arrival ticket must start at zero; the partials are overwritten
  check(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s), "clear dot ticket");
  const int blocks = static_cast<int>(n == 0 ? 1 : (n + kNoAllocChunk - 1) / kNoAllocChunk);
  if (dtype == GS_F32)
    dot_kernel<float><<<blocks, 256, 0, s>>>(static_cast<int>(n), static_cast<const float *>(x), static_cast<const float *>(y), static_cast<float *>(result), partials, ticket);
  else
    dot_kernel<double><<<blocks, 256, 0, s>>>(static_cast<int>(n), static_cast<const double *>(x), static_cast<const double *>(y), static_cast<double *>(result), partials, ticket);
  check(cudaGetLastError(), "dot (no allocation)");
}

void vector_op(int op, long long n, const void *x, void *y, double alpha, const void *alpha_dev,
               int dtype, cudaStream_t s) {
  if (n <= 0) return;
  const int gb = grid_for(n);
  if (dtype == GS_F32)
    vec_kernel<float><<<gb, 256, 0, s>>>(op, n, static_cast<const float *>(x), static_cast<float *>(y), float(alpha), static_cast<const float *>(alpha_dev));
  else
    vec_kernel<double><<<gb, 256, 0, s>>>(op, n, static_cast<const double *>(x), static_cast<double *>(y), alpha, static_cast<const double *>(alpha_dev));
  check(cudaGetLastError(), "vector op");
}

void scalar_op(int op, const void *a, const void *b, void *out, double value, int dtype, cudaStream_t s) {
  if (dtype == GS_F32)
    scalar_kernel<float><<<1, 1, 0, s>>>(op, static_cast<const float *>(a), static_cast<const float *>(b), static_cast<float *>(out), float(value));
  else
    scalar_kernel<double><<<1, 1, 0, s>>>(op, static_cast<const double *>(a), static_cast<const double *>(b), static_cast<double *>(out), value);
  check(cudaGetLastError(), "scalar op");
}

}  // namespace gsb
