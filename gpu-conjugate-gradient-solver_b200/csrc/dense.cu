// Dense inverse of an SPD matrix on the GPU, for coarsest levels too large
// for the host Cholesky (thousands to tens of thousands of rows), in the
// library's own FP64 kernels (setup work; the per-solve dense matvec is
// dense_solve_kernel / dense_tile_kernel).
//
// The CSR matrix is scattered into a dense row-major n x n array (symmetric,
// so it is also its own column-major array). With 64 x 64 tiles (T tiles per
// side, the last one padded with the identity):
//   1. Cholesky A = L L^T, right-looking by tile column k: the diagonal tile
//      is factorised by one CTA in shared memory (which also inverts its
//      factor, L_kk^-1), the panel below becomes A_ik L_kk^-T and every
//      trailing tile (i, j), k < j <= i, loses A_ik A_jk^T.
//   2. Y = L^-1 by forward substitution on the identity, right-looking by
//      tile row i: Y_ic = L_ii^-1 B_ic for c <= i, then B_jc -= L_ji Y_ic for
//      j > i (Y is lower triangular, so only c <= i is carried).
//   3. X = L^-T Y = A^-1 by backward substitution from the last tile row up:
//      X_ic = L_ii^-T B_ic, then B_jc -= L_ij^T X_ic for j < i, c <= j; X is
//      symmetric, so only its lower tiles (c <= i) are formed.
// Every tile product is the same kernel (tile_product_kernel): one CTA per
// output tile, both operand tiles in shared memory, FP64 tensor-core MMAs
// (8 warps, 2 x 4 blocks of 8 x 8 each); each output tile is written by
// exactly one CTA per launch, so the result does not depend on scheduling
// (deterministic).
// A pivot that is not positive (or not finite) marks the matrix "not SPD".
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "dense.h"
#include "solver.h"

namespace gsb {

namespace {

constexpr int kTB = 64;        // tile side
constexpr int kLD = kTB + 1;   // padded shared-memory row (odd stride in doubles)

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// a[i * n + ci[k]] += v[k] for the entries of row i (a zeroed before).
__global__ void csr_scatter_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                   const double *__restrict__ v, double *__restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) a[static_cast<size_t>(i) * n + ci[k]] += v[k];
}

// Row-major lower triangle copied into the upper one.
__global__ void mirror_lower_kernel(int n, double *__restrict__ a) {
  const size_t total = static_cast<size_t>(n) * n;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e / n), j = static_cast<int>(e % n);
    if (j > i) a[e] = a[static_cast<size_t>(j) * n + i];
  }
}

__global__ void identity_kernel(int n, double *__restrict__ a) {
  const size_t total = static_cast<size_t>(n) * n;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x)
    a[e] = (e / n == e % n) ? 1.0 : 0.0;
}

// Tile (ti, tj) of the n x n row-major array into shared memory s[r * kLD + c]
// (transposed: s[c * kLD + r]); entries outside the matrix read as the
// identity's when `eye`, else as zero. 256 threads: each issues its 16
// (coalesced) loads before any store, so one memory latency covers the tile.
constexpr int kLoads = kTB * kTB / 256;

__device__ __forceinline__ void load_tile(const double *__restrict__ a, int n, int ti, int tj, double *s,
                                          bool trans, bool eye) {
  double v[kLoads];
#pragma unroll
  for (int q = 0; q < kLoads; ++q) {
    const int e = threadIdx.x + 256 * q, r = e / kTB, c = e % kTB;
    const int gr = ti * kTB + r, gc = tj * kTB + c;
    v[q] = (gr < n && gc < n) ? a[static_cast<size_t>(gr) * n + gc] : ((eye && gr == gc) ? 1.0 : 0.0);
  }
#pragma unroll
  for (int q = 0; q < kLoads; ++q) {
    const int e = threadIdx.x + 256 * q, r = e / kTB, c = e % kTB;
    if (trans) s[c * kLD + r] = v[q];
    else s[r * kLD + c] = v[q];
  }
}

__device__ __forceinline__ void load_dense_tile(const double *__restrict__ t, double *s, bool trans) {
  double v[kLoads];
#pragma unroll
  for (int q = 0; q < kLoads; ++q) v[q] = t[threadIdx.x + 256 * q];
#pragma unroll
  for (int q = 0; q < kLoads; ++q) {
    const int e = threadIdx.x + 256 * q, r = e / kTB, c = e % kTB;
    if (trans) s[c * kLD + r] = v[q];
    else s[r * kLD + c] = v[q];
  }
}

// ---- 1. the diagonal tile: Cholesky in shared memory and the inverse factor --
// One CTA of 256 threads. L_kk replaces the tile's lower triangle (the strict
// upper triangle is zeroed); L_kk^-1 goes to dinv[k] (64 x 64, row-major,
// identity on the padding of a partial last tile).
__global__ void __launch_bounds__(256) chol_diag_kernel(int n, double *__restrict__ a, int k,
                                                        double *__restrict__ dinv, int *info) {
  extern __shared__ double sm[];
  double *s = sm;                   // the tile, then L
  double *w = sm + kTB * kLD;       // L^-1
  load_tile(a, n, k, k, s, false, true);
  __syncthreads();
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  for (int j = 0; j < kTB; ++j) {
    if (threadIdx.x == 0) {
      double d = s[j * kLD + j];
      if (!(d > 0.0) || !isfinite(d)) {
        bad = 1;
        d = 1.0;  // keep the arithmetic finite; the result is discarded
      }
      s[j * kLD + j] = sqrt(d);
    }
    __syncthreads();
    const double djj = s[j * kLD + j];
    for (int i = j + 1 + threadIdx.x; i < kTB; i += blockDim.x) s[i * kLD + j] /= djj;
    __syncthreads();
    // trailing update of the lower triangle, rows and columns past j
    const int m = kTB - j - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = j + 1 + e / m, l = j + 1 + e % m;
      if (l <= i) s[i * kLD + l] -= s[i * kLD + j] * s[l * kLD + j];
    }
    __syncthreads();
  }
  // L^-1 by columns: thread c solves L w_c = e_c (forward substitution)
  if (threadIdx.x < kTB) {
    const int c = threadIdx.x;
    for (int i = 0; i < kTB; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      if (i >= c) {
        for (int m = c; m < i; ++m) v -= s[i * kLD + m] * w[m * kLD + c];
        v /= s[i * kLD + i];
      } else {
        v = 0.0;
      }
      w[i * kLD + c] = v;
    }
  }
  __syncthreads();
  double *dk = dinv + static_cast<size_t>(k) * kTB * kTB;
  for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
    const int r = e / kTB, c = e % kTB;
    dk[e] = w[r * kLD + c];
    const int gr = k * kTB + r, gc = k * kTB + c;
    if (gr < n && gc < n) a[static_cast<size_t>(gr) * n + gc] = c <= r ? s[r * kLD + c] : 0.0;
  }
  if (threadIdx.x == 0 && bad) atomicExch(info, 1);
}

// ---- 2. every tile product ------------------------------------------------------
enum TileOp : int {
  kPanel = 0,   // step k, tile (k+1+t, k):          C = C L_kk^-T
  kUpdate = 1,  // step k, tiles k < J <= I:          C_IJ -= A_Ik A_Jk^T
  kFwdDiag = 2, // step i, tiles (i, c), c <= i:      C = L_ii^-1 C
  kFwdUpd = 3,  // step i, tiles (j, c), j > i, c <= i: C_jc -= L_ji Y_ic
  kBwdDiag = 4, // step i, tiles (i, c), c <= i:      C = L_ii^-T C
  kBwdUpd = 5,  // step i, tiles (j, c), c <= j < i:  C_jc -= L_ij^T X_ic
};

// (row, col) of task t in the lower triangle 0 <= col <= row (row-major order)
__device__ __forceinline__ void tri_index(long long t, int &row, int &col) {
  int r = static_cast<int>((sqrt(8.0 * static_cast<double>(t) + 1.0) - 1.0) * 0.5);
  while (static_cast<long long>(r) * (r + 1) / 2 > t) --r;
  while (static_cast<long long>(r + 1) * (r + 2) / 2 <= t) ++r;
  row = r;
  col = static_cast<int>(t - static_cast<long long>(r) * (r + 1) / 2);
}

template <int OP>
__global__ void __launch_bounds__(256) tile_product_kernel(int n, int T, int step, double *__restrict__ a,
                                                           double *__restrict__ b, const double *__restrict__ dinv) {
  extern __shared__ double sm[];
  double *sa = sm;               // left operand, sa[m * kLD + kk] = op(X)[m][kk]
  double *sb = sm + kTB * kLD;   // right operand, sb[kk * kLD + j] = op(Y)[kk][j]
  const long long t = blockIdx.x;
  int ci = 0, cj = 0;            // output tile
  double *c = nullptr;           // output array (a or b)
  bool sub = true;
  if (OP == kPanel) {
    ci = step + 1 + static_cast<int>(t), cj = step, c = a, sub = false;
    load_tile(a, n, ci, cj, sa, false, false);
    load_dense_tile(dinv + static_cast<size_t>(step) * kTB * kTB, sb, true);  // (L_kk^-1)^T
  } else if (OP == kUpdate) {
    int r, q;
    tri_index(t, r, q);
    ci = step + 1 + r, cj = step + 1 + q, c = a;
    load_tile(a, n, ci, step, sa, false, false);
    load_tile(a, n, cj, step, sb, true, false);  // A_Jk^T
  } else if (OP == kFwdDiag || OP == kBwdDiag) {
    ci = step, cj = static_cast<int>(t), c = b, sub = false;
    load_dense_tile(dinv + static_cast<size_t>(step) * kTB * kTB, sa, OP == kBwdDiag);
    load_tile(b, n, ci, cj, sb, false, false);
  } else if (OP == kFwdUpd) {
    const int w = step + 1;
    ci = step + 1 + static_cast<int>(t / w), cj = static_cast<int>(t % w), c = b;
    load_tile(a, n, ci, step, sa, false, false);   // L_ji
    load_tile(b, n, step, cj, sb, false, false);   // Y_ic
  } else {  // kBwdUpd
    int r, q;
    tri_index(t, r, q);
    ci = r, cj = q, c = b;
    load_tile(a, n, step, ci, sa, true, false);    // L_ij^T
    load_tile(b, n, step, cj, sb, false, false);   // X_ic
  }
  __syncthreads();
  // FP64 tensor-core products (mma.sync m8n8k4, the only FP64 MMA shape):
  // warp w owns rows 16 (w / 2) .. +16 and columns 32 (w % 2) .. +32 of the
  // output tile, as 2 x 4 blocks of 8 x 8. Fragments: A (8 x 4, row-major)
  // element (lane / 4, lane % 4); B (4 x 8, column-major) element
  // (lane % 4, lane / 4); C/D (8 x 8) elements (lane / 4, 2 (lane % 4) + {0, 1}).
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = (w >> 1) * 16, n0 = (w & 1) * 32;
  const int fr = lane >> 2, fc = lane & 3;
  double acc[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
  for (int kk = 0; kk < kTB; kk += 4) {
    double fa[2], fb[4];
#pragma unroll
    for (int i = 0; i < 2; ++i) fa[i] = sa[(m0 + 8 * i + fr) * kLD + kk + fc];
#pragma unroll
    for (int j = 0; j < 4; ++j) fb[j] = sb[(kk + fc) * kLD + n0 + 8 * j + fr];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                     : "d"(fa[i]), "d"(fb[j]));
  }
  // every CTA owns its output tile: read-modify-write without races (all
  // 16 old values are requested before any is written back)
  double old[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int gr = ci * kTB + m0 + 8 * i + fr, gc = cj * kTB + n0 + 8 * j + 2 * fc + q;
        old[i][j][q] = (sub && gr < n && gc < n) ? c[static_cast<size_t>(gr) * n + gc] : 0.0;
      }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int gr = ci * kTB + m0 + 8 * i + fr, gc = cj * kTB + n0 + 8 * j + 2 * fc + q;
        if (gr < n && gc < n) c[static_cast<size_t>(gr) * n + gc] = sub ? old[i][j][q] - acc[i][j][q] : acc[i][j][q];
      }
  (void)T;
}

template <int OP>
void launch_tiles(long long tasks, int n, int T, int step, double *a, double *b, const double *dinv,
                  cudaStream_t s) {
  if (tasks <= 0) return;
  const size_t smem = 2 * kTB * kLD * sizeof(double);
  check(cudaFuncSetAttribute(tile_product_kernel<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)),
        "dense tile product attribute");
  if (tasks > 0x7fffffffLL) throw std::runtime_error("dense inverse: too many tiles");
  tile_product_kernel<OP><<<static_cast<unsigned>(tasks), 256, smem, s>>>(n, T, step, a, b, dinv);
  check(cudaGetLastError(), "dense tile product");
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

void spd_inverse_device(const Csr &m, double *d_out, cudaStream_t s, bool lower_only) {
  const int n = m.rows;
  if (m.cols != n) throw std::runtime_error("dense inverse: matrix must be square");
  if (n == 0) return;
  const size_t total = static_cast<size_t>(n) * n;
  const int T = (n + kTB - 1) / kTB;
  DevArray<int> rp(m.rp.size()), ci(m.ci.size()), info(1);
  DevArray<double> v(m.v.size()), a(total), dinv(static_cast<size_t>(T) * kTB * kTB);
  check(cudaMemcpyAsync(rp.p, m.rp.data(), sizeof(int) * m.rp.size(), cudaMemcpyHostToDevice, s), "dense upload");
  if (!m.ci.empty()) {
    check(cudaMemcpyAsync(ci.p, m.ci.data(), sizeof(int) * m.ci.size(), cudaMemcpyHostToDevice, s), "dense upload");
    check(cudaMemcpyAsync(v.p, m.v.data(), sizeof(double) * m.v.size(), cudaMemcpyHostToDevice, s), "dense upload");
  }
  check(cudaMemsetAsync(info.p, 0, sizeof(int), s), "dense info");
  check(cudaMemsetAsync(a.p, 0, sizeof(double) * total, s), "dense zero");
  csr_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, rp.p, ci.p, v.p, a.p);
  check(cudaGetLastError(), "dense scatter");
  const size_t smem = 2 * kTB * kLD * sizeof(double);
  check(cudaFuncSetAttribute(chol_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
        "dense diag attribute");
  // 1. A = L L^T
  for (int k = 0; k < T; ++k) {
    chol_diag_kernel<<<1, 256, smem, s>>>(n, a.p, k, dinv.p, info.p);
    check(cudaGetLastError(), "dense diagonal tile");
    const long long below = T - k - 1;
    launch_tiles<kPanel>(below, n, T, k, a.p, nullptr, dinv.p, s);
    launch_tiles<kUpdate>(below * (below + 1) / 2, n, T, k, a.p, nullptr, dinv.p, s);
  }
  int hinfo = 0;
  check(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s), "dense info");
  check(cudaStreamSynchronize(s), "dense factorisation");
  if (hinfo != 0) throw std::runtime_error("coarsest level matrix is not SPD (Cholesky failed)");
  // 2. Y = L^-1 (into d_out, from the identity)
  const int grid = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
  identity_kernel<<<grid, 256, 0, s>>>(n, d_out);
  check(cudaGetLastError(), "dense identity");
  for (int i = 0; i < T; ++i) {
    launch_tiles<kFwdDiag>(i + 1, n, T, i, a.p, d_out, dinv.p, s);
    launch_tiles<kFwdUpd>(static_cast<long long>(T - i - 1) * (i + 1), n, T, i, a.p, d_out, dinv.p, s);
  }
  // 3. X = L^-T Y, lower tiles
  for (int i = T - 1; i >= 0; --i) {
    launch_tiles<kBwdDiag>(i + 1, n, T, i, a.p, d_out, dinv.p, s);
    launch_tiles<kBwdUpd>(static_cast<long long>(i) * (i + 1) / 2, n, T, i, a.p, d_out, dinv.p, s);
  }
  if (!lower_only) {
    mirror_lower_kernel<<<grid, 256, 0, s>>>(n, d_out);
    check(cudaGetLastError(), "dense mirror");
  }
  check(cudaStreamSynchronize(s), "dense inverse");
}

int dense_depth(const std::vector<int> &level_rows, int coarse_rows) {
  const int L = static_cast<int>(level_rows.size());
  if (coarse_rows <= 0) return L;
  for (int k = 1; k < L; ++k)
    if (level_rows[k] <= coarse_rows) return k + 1;
  return L;
}

}  // namespace gsb
