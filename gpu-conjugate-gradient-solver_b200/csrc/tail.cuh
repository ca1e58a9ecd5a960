// The coarse tail of the V-cycle in one launch.
//
// The smallest levels of the hierarchy carry little work per colour pass
// (tens to a few hundred rows) but many passes (Galerkin operators colour
// into 30-50 colours, four sweeps per V-cycle), so one kernel per pass leaves
// the GPU idle between launches, and even a single resident kernel is bound
// by the latency of each pass's dependent loads (row pointer -> column ->
// x gather). Here one thread-block cluster (up to 16 CTAs of 1024 threads,
// co-scheduled by the hardware) walks the whole V-cycle of levels k0..L-1 --
// pre-smoothing, residual, restriction, the coarsest solve, prolongation,
// post-smoothing -- with these properties:
//   * every CTA keeps a full replica of each tail level's iterate x in its
//     shared memory; a thread that updates x[row] writes the new value into
//     all replicas of the cluster (distributed shared memory), so every
//     gather is a local shared-memory read;
//   * a thread keeps the same rows in every pass (static assignment), so its
//     slice of the level matrices stays resident in its SM's L1 after the
//     first sweep (read-only path);
//   * dependent steps are separated by the cluster barrier
//     (barrier.cluster.arrive.release / wait.acquire): no software spin-wait.
//     Global vectors written by other CTAs (b, r) are read through L2
//     (ld.global.cg), never from a possibly stale L1 line.
// Semantics are those of the per-pass kernels (same colouring, same update
// formula, same zero-initial-guess handling); results match the multi-launch
// V-cycle up to the order of floating-point summation.
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace gsb {

template <typename T>
struct TailLevel {
  int n = 0, ncolors = 0;
  int g = 32, rg = 32, pg = 8;      // lanes per row for A, R (to the next level), P (from it)
  int xoff = 0;                     // offset of this level's x replica in shared memory (elements)
  const int *color_first = nullptr; // ncolors + 1, device
  const T *wts = nullptr;           // per-colour weights (device) or nullptr
  CsrvView<T> A{}, R{}, P{};        // R, P: to / from level k+1
  T *x = nullptr, *b = nullptr, *r = nullptr;
  const T *ainv = nullptr;          // coarsest dense inverse, or nullptr
};

template <typename T>
struct TailParams {
  int k0, L;                 // levels k0..L-1 (L-1 is the coarsest), k0 >= 1
  int pre, post, coarse_steps;
  int coarse_dense;          // 1: dense solve on L-1; 0: smoother steps
  int alias;                 // 1: reference V-cycle (x_k = 2 P x_{k+1} below the finest)
  T omega;
  const TailLevel<T> *lv;    // device array indexed by level
};

namespace tail_detail {

// Writes v into x[row] of every CTA's replica.
template <typename T>
__device__ __forceinline__ void broadcast(cooperative_groups::cluster_group &cl, T *xs, int row, T v) {
  const unsigned nb = cl.num_blocks();
  for (unsigned q = 0; q < nb; ++q) *cl.map_shared_rank(xs + row, q) = v;
}

// Off-diagonal row sum with g lanes per row; x is a shared-memory replica.
template <typename T>
__device__ __forceinline__ T row_offdiag(const CsrvView<T> &A, int row, bool valid, int sub, int g,
                                         const T *xs, int skip_from) {
  T sum = T(0);
  if (valid) {
    const int k1 = __ldg(A.rp + row + 1);
    for (int k = __ldg(A.rp + row) + sub; k < k1; k += g) {
      const int c = __ldg(A.ci + k);
      if (c < skip_from) sum = fma(__ldg(A.v + k), xs[c], sum);
    }
  }
  for (int o = g >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, g);
  return sum;
}

// One GS colour pass over rows [r0, r1); `zero`: x is an implicit zero
// vector (first forward sweep from a zero guess).
template <typename T>
__device__ void gs_pass(cooperative_groups::cluster_group &cl, const TailLevel<T> &L, T *xs, int c,
                        bool zero, T omega, int tid, int nthr) {
  const int r0 = L.color_first[c], r1 = L.color_first[c + 1];
  const int g = L.g, sub = tid & (g - 1), groups = nthr / g;
  const int trips = (r1 - r0 + groups - 1) / groups;
  const T w = L.wts != nullptr ? L.wts[c] : omega;
  for (int t = 0; t < trips; ++t) {
    const int row = r0 + tid / g + t * groups;
    const bool valid = row < r1;
    const T off = row_offdiag(L.A, row, valid, sub, g, xs, zero ? r0 : 0x7fffffff);
    if (valid && sub == 0) {
      const T gs = (__ldcg(L.b + row) - off) / __ldg(L.A.diag + row);
      broadcast(cl, xs, row, zero ? w * gs : (T(1) - w) * xs[row] + w * gs);
    }
  }
}

template <typename T>
__device__ void smooth(cooperative_groups::cluster_group &cl, const TailLevel<T> &L, T *xs, int steps,
                       bool zero, T omega, int tid, int nthr) {
  for (int s = 0; s < steps; ++s) {
    for (int c = 0; c < L.ncolors; ++c) {
      gs_pass(cl, L, xs, c, zero && s == 0, omega, tid, nthr);
      cl.sync();
    }
    for (int c = L.ncolors - 1; c >= 0; --c) {
      gs_pass(cl, L, xs, c, false, omega, tid, nthr);
      cl.sync();
    }
  }
}

}  // namespace tail_detail

template <typename T>
__global__ void __launch_bounds__(1024, 1) coarse_tail_kernel(TailParams<T> p, const int *done) {
  namespace cg = cooperative_groups;
  using namespace tail_detail;
  extern __shared__ __align__(16) unsigned char tail_smem[];
  T *smem = reinterpret_cast<T *>(tail_smem);
  cg::cluster_group cl = cg::this_cluster();
  // uniform across the cluster: every CTA returns or none does
  if (stop_requested(done)) return;
  const int tid = static_cast<int>(cl.thread_rank());
  const int nthr = static_cast<int>(cl.num_threads());
  // down: pre-smoothing, residual, restriction
  for (int k = p.k0; k < p.L - 1; ++k) {
    const TailLevel<T> &L = p.lv[k];
    T *xs = smem + L.xoff;
    smooth(cl, L, xs, p.pre, true, p.omega, tid, nthr);
    {  // r = b - A x
      const int g = L.g, sub = tid & (g - 1), groups = nthr / g;
      const int trips = (L.n + groups - 1) / groups;
      for (int t = 0; t < trips; ++t) {
        const int row = tid / g + t * groups;
        const bool valid = row < L.n;
        const T off = row_offdiag(L.A, row, valid, sub, g, xs, 0x7fffffff);
        if (valid && sub == 0) L.r[row] = __ldcg(L.b + row) - fma(__ldg(L.A.diag + row), xs[row], off);
      }
    }
    cl.sync();
    {  // b_{k+1} = R r (R's columns index level k; r is read through L2)
      const TailLevel<T> &C = p.lv[k + 1];
      const int g = L.rg, sub = tid & (g - 1), groups = nthr / g;
      const int trips = (C.n + groups - 1) / groups;
      for (int t = 0; t < trips; ++t) {
        const int row = tid / g + t * groups;
        const bool valid = row < C.n;
        T sum = T(0);
        if (valid) {
          const int k1 = __ldg(L.R.rp + row + 1);
          for (int q = __ldg(L.R.rp + row) + sub; q < k1; q += g)
            sum = fma(__ldg(L.R.v + q), __ldcg(L.r + __ldg(L.R.ci + q)), sum);
        }
        for (int o = g >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, g);
        if (valid && sub == 0) C.b[row] = sum;
      }
    }
    cl.sync();
  }
  {  // coarsest level
    const TailLevel<T> &C = p.lv[p.L - 1];
    T *xs = smem + C.xoff;
    if (p.coarse_dense) {
      const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
      for (int row = warp; row < C.n; row += nwarps) {
        const T *a = C.ainv + static_cast<size_t>(row) * C.n;
        double sum = 0.0;
        for (int j = lane; j < C.n; j += 32) sum = fma(double(__ldg(a + j)), double(__ldcg(C.b + j)), sum);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (lane == 0) broadcast(cl, xs, row, T(sum));
      }
      cl.sync();
    } else {
      smooth(cl, C, xs, p.coarse_steps, true, p.omega, tid, nthr);
    }
  }
  // up: x_k += P x_{k+1} (or x_k = 2 P x_{k+1}), post-smoothing
  for (int k = p.L - 2; k >= p.k0; --k) {
    const TailLevel<T> &L = p.lv[k];
    T *xs = smem + L.xoff;
    const T *xc = smem + p.lv[k + 1].xoff;
    {
      const int g = L.pg, sub = tid & (g - 1), groups = nthr / g;
      const int trips = (L.n + groups - 1) / groups;
      for (int t = 0; t < trips; ++t) {
        const int row = tid / g + t * groups;
        const bool valid = row < L.n;
        const T sum = row_offdiag(L.P, row, valid, sub, g, xc, 0x7fffffff);
        if (valid && sub == 0) broadcast(cl, xs, row, p.alias ? sum + sum : xs[row] + sum);
      }
    }
    cl.sync();
    smooth(cl, L, xs, p.post, false, p.omega, tid, nthr);
  }
  {  // hand x_{k0} back to the per-pass launches above the tail
    const TailLevel<T> &L = p.lv[p.k0];
    const T *xs = smem + L.xoff;
    for (int row = tid; row < L.n; row += nthr) L.x[row] = xs[row];
  }
}

}  // namespace gsb
