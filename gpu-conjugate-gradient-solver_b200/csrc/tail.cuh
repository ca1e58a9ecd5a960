// The coarse tail of the V-cycle in one launch.
//
// Below some size the levels of the hierarchy carry little work per colour
// pass (tens to a few thousand rows) but many passes (Galerkin operators
// colour into 30-50 colours, four sweeps per V-cycle), so launching one
// kernel per pass leaves the GPU mostly idle between launches. Here one
// thread-block cluster (up to 16 CTAs of 1024 threads, co-scheduled by the
// hardware) walks the whole V-cycle of levels k0..L-1 -- pre-smoothing,
// residual, restriction, the coarsest solve, prolongation, post-smoothing --
// and separates dependent steps with the cluster barrier
// (barrier.cluster.arrive.release / wait.acquire). There is no software
// spin-wait. Vectors written by other CTAs of the cluster are read through
// L2 (ld.global.cg) so no stale L1 line is ever used; the read-only level
// matrices go through the read-only path.
//
// Semantics are exactly those of the per-pass kernels (same colouring, same
// update formula, same zero-initial-guess handling), so results match the
// multi-launch V-cycle up to the order of floating-point summation.
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace gsb {

template <typename T>
struct TailLevel {
  int n = 0, ncolors = 0;
  int g = 32, rg = 32, pg = 8;     // lanes per row for A, R (to the next level), P (from it)
  const int *color_first = nullptr; // ncolors + 1, device
  const T *wts = nullptr;           // per-colour weights (device) or nullptr
  CsrvView<T> A{}, R{}, P{};        // R, P: to / from level k+1
  T *x = nullptr, *b = nullptr, *r = nullptr;
  const double *ainv = nullptr;     // coarsest dense inverse, or nullptr
};

template <typename T>
struct TailParams {
  int k0, L;                 // levels k0..L-1 (L-1 is the coarsest)
  int pre, post, coarse_steps;
  int coarse_dense;          // 1: dense solve on L-1; 0: smoother steps
  int alias;                 // 1: reference V-cycle (x_k = 2 P x_{k+1} below the finest; k0 >= 1)
  T omega;
  const TailLevel<T> *lv;    // device array indexed by level
};

namespace tail_detail {

template <typename T>
__device__ __forceinline__ T row_offdiag(const CsrvView<T> &A, int row, bool valid, int sub, int g,
                                         const T *x, int skip_from) {
  T sum = T(0);
  if (valid) {
    const int k1 = __ldg(A.rp + row + 1);
    for (int k = __ldg(A.rp + row) + sub; k < k1; k += g) {
      const int c = __ldg(A.ci + k);
      if (c < skip_from) sum = fma(__ldg(A.v + k), __ldcg(x + c), sum);
    }
  }
  for (int o = g >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, g);
  return sum;
}

// One GS colour pass over rows [r0, r1) with g lanes per row; `zero`: x is
// an implicit zero vector (first forward sweep from a zero guess).
template <typename T>
__device__ void gs_pass(const TailLevel<T> &L, int c, bool zero, T omega, int tid, int nthr) {
  const int r0 = L.color_first[c], r1 = L.color_first[c + 1];
  const int g = L.g, sub = tid & (g - 1), groups = nthr / g;
  const int trips = (r1 - r0 + groups - 1) / groups;
  const T w = L.wts != nullptr ? L.wts[c] : omega;
  for (int t = 0; t < trips; ++t) {
    const int row = r0 + tid / g + t * groups;
    const bool valid = row < r1;
    const T off = row_offdiag(L.A, row, valid, sub, g, L.x, zero ? r0 : 0x7fffffff);
    if (valid && sub == 0) {
      const T gs = (__ldcg(L.b + row) - off) / L.A.diag[row];
      L.x[row] = zero ? w * gs : (T(1) - w) * __ldcg(L.x + row) + w * gs;
    }
  }
}

// y = b - A x (mode 1), y = A x (0), y += A x (2), y = 2 A x (3).
template <typename T>
__device__ void spmv(const CsrvView<T> &A, int g, const T *x, T *y, const T *b, int mode, int tid,
                     int nthr) {
  const int sub = tid & (g - 1), groups = nthr / g;
  const int trips = (A.rows + groups - 1) / groups;
  for (int t = 0; t < trips; ++t) {
    const int row = tid / g + t * groups;
    const bool valid = row < A.rows;
    T sum = row_offdiag(A, row, valid, sub, g, x, 0x7fffffff);
    if (valid && sub == 0) {
      if (A.diag != nullptr) sum = fma(A.diag[row], __ldcg(x + row), sum);
      if (mode == 0) y[row] = sum;
      else if (mode == 1) y[row] = __ldcg(b + row) - sum;
      else if (mode == 2) y[row] = __ldcg(y + row) + sum;
      else y[row] = sum + sum;
    }
  }
}

template <typename T>
__device__ void smooth(const TailLevel<T> &L, int steps, bool zero, T omega, int tid, int nthr,
                       cooperative_groups::cluster_group &cl) {
  for (int s = 0; s < steps; ++s) {
    for (int c = 0; c < L.ncolors; ++c) {
      gs_pass(L, c, zero && s == 0, omega, tid, nthr);
      cl.sync();
    }
    for (int c = L.ncolors - 1; c >= 0; --c) {
      gs_pass(L, c, false, omega, tid, nthr);
      cl.sync();
    }
  }
}

}  // namespace tail_detail

template <typename T>
__global__ void __launch_bounds__(1024, 1) coarse_tail_kernel(TailParams<T> p, const int *done) {
  namespace cg = cooperative_groups;
  using namespace tail_detail;
  cg::cluster_group cl = cg::this_cluster();
  // uniform across the cluster: every CTA returns or none does
  if (stop_requested(done)) return;
  const int tid = static_cast<int>(cl.thread_rank());
  const int nthr = static_cast<int>(cl.num_threads());
  // down
  for (int k = p.k0; k < p.L - 1; ++k) {
    const TailLevel<T> &L = p.lv[k];
    smooth(L, p.pre, true, p.omega, tid, nthr, cl);
    spmv(L.A, L.g, L.x, L.r, L.b, 1, tid, nthr);
    cl.sync();
    spmv(L.R, L.rg, L.r, p.lv[k + 1].b, static_cast<const T *>(nullptr), 0, tid, nthr);
    cl.sync();
  }
  // coarsest
  {
    const TailLevel<T> &C = p.lv[p.L - 1];
    if (p.coarse_dense) {
      const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
      for (int row = warp; row < C.n; row += nwarps) {
        const double *a = C.ainv + static_cast<size_t>(row) * C.n;
        double sum = 0.0;
        for (int j = lane; j < C.n; j += 32) sum = fma(__ldg(a + j), double(__ldcg(C.b + j)), sum);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (lane == 0) C.x[row] = T(sum);
      }
      cl.sync();
    } else {
      smooth(C, p.coarse_steps, true, p.omega, tid, nthr, cl);
    }
  }
  // up
  for (int k = p.L - 2; k >= p.k0; --k) {
    const TailLevel<T> &L = p.lv[k];
    spmv(L.P, L.pg, p.lv[k + 1].x, L.x, static_cast<const T *>(nullptr), p.alias ? 3 : 2, tid, nthr);
    cl.sync();
    smooth(L, p.post, false, p.omega, tid, nthr, cl);
  }
}

}  // namespace gsb
