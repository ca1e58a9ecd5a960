// Whole symmetric Gauss-Seidel sweeps of one level in ONE cooperative launch.
//
// A multicolour sweep is a chain of colour passes, each depending on the one
// before. On the coarse Galerkin levels a pass is short (a few thousand rows,
// long rows) and latency-bound, so launching one kernel per colour costs a
// launch, a drain and a cold start per pass (the reference's structure,
// src/Smoothers/SymmetricGaussSeidelSmoother.cc:80-128: one launch per colour).
// Here every block of a cooperative grid (all co-resident, guaranteed by
// the launch) walks the same pass list and meets the others at a grid barrier
// between passes. Before it waits at a barrier each thread already loads the
// operands of its next row (or slice) that do not depend on the iterate --
// the slice/row bounds, the first column indices and values, the diagonal and
// the right-hand side -- so only the neighbour gathers and the update remain
// after the barrier opens.
//
// Each row is updated with exactly the arithmetic of the per-colour kernels
// (sell_gs_kernel / csrv_gs_kernel: same head loads, same summation order,
// same shuffles), so iterates are bit-identical to one launch per colour.
// The iterate is read through L2 (ld.global.cg): other SMs write it inside
// the same launch, and the L1 of this SM may hold an older copy.
//
// Every barrier wait is bounded: after kSweepSpinLimit polls a block gives up,
// records the fault in CgState::sync_fault, stops the solve (done) and leaves;
// every later wait of the launch gives up at once. The host turns the flag
// into an error and clears the barrier state. With the cooperative launch
// all blocks are resident, so the limit is never reached in a correct run.
#pragma once

#include "kernels.cuh"

namespace gsb {

constexpr int kSweepThreads = 1024;               // one block per SM
constexpr unsigned kSweepSpinLimit = 1u << 21;    // ~1-2 s of polling

// Barrier state of one solver's cooperative launches (device memory, zero
// between launches: the last block to leave a launch resets it).
struct SweepSync {
  unsigned int arrive;  // arrivals in this launch; barrier k opens at k * gridDim.x
  unsigned int leave;   // blocks that finished this launch
};

// The passes of `steps` symmetric steps (forward colours 0..C-1, backward
// C-1..0, per step) over unit ranges bounds[c] .. bounds[c+1] (slices of the
// sliced layout, rows of the CSR-vector layout); first_row[c] is the first
// row of colour c (the zero-guess skip bound).
struct SweepPlan {
  const int *bounds;
  const int *first_row;
  int ncolors, steps;
  int zero;    // x is an implicit zero before the first forward pass
  int skip;    // drop a pass whose colour equals the previous pass's colour
  int forward_only;  // one forward sweep (timing), no backward passes
};

__device__ __forceinline__ int sweep_passes(const SweepPlan &p) {
  return p.forward_only ? p.ncolors : 2 * p.ncolors * p.steps;
}

// Colour of pass q; -1 if the plan drops it. With omega = 1 and no learned
// weight the repeated colour at a direction change is an exact no-op (the
// update does not depend on the row's own value and its neighbours did not
// change), so it is skipped.
__device__ __forceinline__ int sweep_colour(const SweepPlan &p, int q, bool &zero_pass) {
  const int C = p.ncolors;
  zero_pass = false;
  if (p.forward_only) {
    zero_pass = p.zero != 0;
    return q;
  }
  const int s = q / (2 * C), r = q % (2 * C);
  if (p.skip && (r == C || (r == 0 && s > 0))) return -1;
  zero_pass = p.zero != 0 && s == 0 && r < C;
  return r < C ? r : 2 * C - 1 - r;
}

__device__ __forceinline__ int sweep_next(const SweepPlan &p, int q, int total, int &colour, bool &zero_pass) {
  for (++q; q < total; ++q) {
    colour = sweep_colour(p, q, zero_pass);
    if (colour >= 0) return q;
  }
  return total;
}

__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void red_relaxed_gpu_add(unsigned *p, unsigned v) {
  asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier number k (1, 2, ...) of this launch; bounded (see above).
// Release: the block's writes, gathered by bar.sync, are ordered before the
// arrival by a gpu-scope fence (fence-based release pattern). Acquire: the
// arrival count is polled with relaxed loads and a gpu-scope fence follows
// the poll that saw it complete (fence-based acquire pattern).
__device__ __forceinline__ void sweep_barrier(SweepSync *sy, CgState *st, unsigned k) {
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_acq_rel_gpu();
    red_relaxed_gpu_add(&sy->arrive, 1u);
    const unsigned target = k * gridDim.x;
    if (*reinterpret_cast<volatile int *>(&st->sync_fault) == 0) {
      unsigned spins = 0;
      while (ld_relaxed_gpu(&sy->arrive) < target) {
        if (++spins >= kSweepSpinLimit) {
          atomicExch(&st->sync_fault, 1);
          atomicExch(&st->done, 1);
          break;
        }
        if ((spins & 63u) == 0 && *reinterpret_cast<volatile int *>(&st->sync_fault) != 0) break;
        if (spins > 2048) __nanosleep(128);
      }
    }
    fence_acq_rel_gpu();
  }
  __syncthreads();
}

__device__ __forceinline__ void sweep_leave(SweepSync *sy) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned left = atomicAdd(&sy->leave, 1u);
    if (left == gridDim.x - 1) {  // every block is past every barrier
      atomicExch(&sy->arrive, 0u);
      atomicExch(&sy->leave, 0u);
    }
  }
}

template <typename T>
__device__ __forceinline__ T ld_l2(const T *p) {
  return __ldcg(p);
}

// ---- CSR-vector layout, G lanes per row ---------------------------------------
// The neighbour sum of csrv_offdiag_head with the iterate read through L2.
template <typename T, bool kSkip, int G>
__device__ __forceinline__ T csrv_offdiag_head_l2(const CsrvView<T> &A, const CsrvHead<T, 8> &h,
                                                  const T *x, int skip_from) {
  constexpr int kE = 8;
  T sum = T(0);
  {
    T xv[kE];
#pragma unroll
    for (int u = 0; u < kE; ++u) {
      const bool use = h.c[u] >= 0 && (!kSkip || h.c[u] < skip_from);
      xv[u] = use ? ld_l2(x + h.c[u]) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kE; ++u) sum = fma(h.v[u], xv[u], sum);
  }
  for (int k0 = h.k0 + kE * G; k0 < h.k1; k0 += 4 * G) {
    int c[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) c[u] = k0 + u * G < h.k1 ? __ldg(A.ci + k0 + u * G) : -1;
    T xv[4], v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool use = c[u] >= 0 && (!kSkip || c[u] < skip_from);
      xv[u] = use ? ld_l2(x + c[u]) : T(0);
      v[u] = c[u] >= 0 ? __ldg(A.v + k0 + u * G) : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) sum = fma(v[u], xv[u], sum);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
  return sum;
}

// Operands of one row that do not depend on the iterate.
template <typename T, typename BT>
struct CsrvRowPre {
  CsrvHead<T, 8> h;
  T di, bi;
};

template <typename T, typename BT, int G>
__device__ __forceinline__ void csrv_row_pre(const CsrvView<T> &A, const BT *b, int row, bool valid, int sub,
                                             CsrvRowPre<T, BT> &p) {
  csrv_head<T, G>(A, row, valid, sub, p.h);
  p.di = valid && sub == 0 ? __ldg(A.diag + row) : T(1);
  p.bi = valid && sub == 0 ? T(__ldg(b + row)) : T(0);
}

template <typename T, typename BT, bool kZero, int G>
__device__ __forceinline__ void csrv_row_update(const CsrvView<T> &A, const CsrvRowPre<T, BT> &p, int row,
                                                bool valid, int sub, T *x, T w, int row_begin) {
  T xi = T(0);
  if (!kZero && valid && sub == 0) xi = ld_l2(x + row);
  const T off = csrv_offdiag_head_l2<T, kZero, G>(A, p.h, x, row_begin);
  if (valid && sub == 0) {
    const T gs = (p.bi - off) / p.di;
    x[row] = kZero ? w * gs : (T(1) - w) * xi + w * gs;
  }
}

template <typename T, typename BT, int G>
__global__ void __launch_bounds__(kSweepThreads, 1) csrv_sweep_kernel(CsrvView<T> A, SweepPlan plan,
                                                                      const BT *__restrict__ b, T *x,
                                                                      const T *__restrict__ wts, T omega,
                                                                      CgState *st, SweepSync *sy) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (stop_requested(&st->done)) return;  // uniform: nothing else writes done during this launch
  // Warps are numbered across blocks first (warp w of block b is number
  // w * gridDim.x + b), so every colour, however short, is spread over all
  // SMs; a warp serves 32 / G consecutive rows.
  const int sub = threadIdx.x & (G - 1);
  const int groups = (gridDim.x * blockDim.x) / G;
  const int gid = (((threadIdx.x >> 5) * gridDim.x + blockIdx.x) << 5 | (threadIdx.x & 31)) / G;
  const int total = sweep_passes(plan);
  bool zero = false;
  int c = -1;
  int q = sweep_next(plan, -1, total, c, zero);
  CsrvRowPre<T, BT> pre;
  if (q < total) {
    const int r0 = plan.bounds[c], r1 = plan.bounds[c + 1];
    csrv_row_pre<T, BT, G>(A, b, r0 + gid, r0 + gid < r1, sub, pre);
  }
  unsigned barrier = 0;
  while (q < total) {
    const int r0 = plan.bounds[c], r1 = plan.bounds[c + 1];
    const T w = wts != nullptr ? wts[c] : omega;
    const int trips = (r1 - r0 + groups - 1) / groups;  // uniform over the warp
    for (int t = 0; t < trips; ++t) {
      const int row = r0 + gid + t * groups;
      const bool valid = row < r1;
      if (t > 0) csrv_row_pre<T, BT, G>(A, b, row, valid, sub, pre);
      if (zero) csrv_row_update<T, BT, true, G>(A, pre, row, valid, sub, x, w, r0);
      else csrv_row_update<T, BT, false, G>(A, pre, row, valid, sub, x, w, r0);
    }
    int cn = -1;
    bool zn = false;
    const int qn = sweep_next(plan, q, total, cn, zn);
    if (qn < total) {
      const int n0 = plan.bounds[cn], n1 = plan.bounds[cn + 1];
      csrv_row_pre<T, BT, G>(A, b, n0 + gid, n0 + gid < n1, sub, pre);
      sweep_barrier(sy, st, ++barrier);
    }
    q = qn, c = cn, zero = zn;
  }
  sweep_leave(sy);
}

// ---- sliced layout (SELL-G), one warp per slice -----------------------------------
template <typename T, bool kSkip>
__device__ __forceinline__ T sell_offdiag_head_l2(const SellView<T> &A, const SellHead<T> &h, int lane,
                                                  const T *x, int skip_from) {
  using P2 = typename Pair<T>::type;
  constexpr int kP = SellHead<T>::kPairs;
  P2 vn;
  int2 cn = make_int2(-1, -1);
  vn.x = vn.y = T(0);
  const int pn = h.p0 + 64 * kP + 2 * lane;
  if (pn < h.p1) {
    vn = __ldg(reinterpret_cast<const P2 *>(A.val + pn));
    cn = __ldg(reinterpret_cast<const int2 *>(A.col + pn));
  }
  T g[2 * kP + 2];
#pragma unroll
  for (int q = 0; q < kP; ++q) {
    const bool ok0 = h.c[q].x >= 0 && (!kSkip || h.c[q].x < skip_from);
    const bool ok1 = h.c[q].y >= 0 && (!kSkip || h.c[q].y < skip_from);
    g[2 * q] = ok0 ? ld_l2(x + h.c[q].x) : T(0);
    g[2 * q + 1] = ok1 ? ld_l2(x + h.c[q].y) : T(0);
  }
  {
    const bool ok0 = cn.x >= 0 && (!kSkip || cn.x < skip_from);
    const bool ok1 = cn.y >= 0 && (!kSkip || cn.y < skip_from);
    g[2 * kP] = ok0 ? ld_l2(x + cn.x) : T(0);
    g[2 * kP + 1] = ok1 ? ld_l2(x + cn.y) : T(0);
  }
  T sum = T(0);
#pragma unroll
  for (int q = 0; q < kP; ++q) {
    sum = fma(h.v[q].x, g[2 * q], sum);
    sum = fma(h.v[q].y, g[2 * q + 1], sum);
  }
  sum = fma(vn.x, g[2 * kP], sum);
  sum = fma(vn.y, g[2 * kP + 1], sum);
  for (int p = pn + 64; p < h.p1; p += 64) {
    const P2 v = __ldg(reinterpret_cast<const P2 *>(A.val + p));
    const int2 c = __ldg(reinterpret_cast<const int2 *>(A.col + p));
    if (!kSkip || c.x < skip_from) sum = fma(v.x, ld_l2(x + c.x), sum);
    if (!kSkip || c.y < skip_from) sum = fma(v.y, ld_l2(x + c.y), sum);
  }
  return sum;
}

template <typename T, typename BT>
struct SellSlicePre {
  SellHead<T> h;
  T di, bi;
};

template <typename T, typename BT, int G>
__device__ __forceinline__ void sell_slice_pre(const SellView<T> &A, const BT *b, int s, bool valid_slice,
                                               int lane, SellSlicePre<T, BT> &p) {
  p.di = T(1);
  p.bi = T(0);
  if (!valid_slice) {
    p.h.r0 = p.h.r1 = p.h.p0 = p.h.p1 = 0;
    return;
  }
  p.di = sell_head<T, G>(A, s, lane, p.h);
  const int row = p.h.r0 + lane / G;
  if ((lane & (G - 1)) == 0 && row < p.h.r1) p.bi = T(__ldg(b + row));
}

template <typename T, typename BT, bool kZero, int G>
__device__ __forceinline__ void sell_slice_update(const SellView<T> &A, const SellSlicePre<T, BT> &p, int lane,
                                                  T *x, T w, int row_begin) {
  const int row = p.h.r0 + lane / G;
  const bool valid = (lane & (G - 1)) == 0 && row < p.h.r1;
  T xi = T(0);
  if (!kZero && valid) xi = ld_l2(x + row);
  T off = sell_offdiag_head_l2<T, kZero>(A, p.h, lane, x, row_begin);
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
  if (valid) {
    const T gs = (p.bi - off) / p.di;
    x[row] = kZero ? w * gs : (T(1) - w) * xi + w * gs;
  }
}

template <typename T, typename BT, int G>
__global__ void __launch_bounds__(kSweepThreads, 1) sell_sweep_kernel(SellView<T> A, SweepPlan plan,
                                                                      const BT *__restrict__ b, T *x,
                                                                      const T *__restrict__ wts, T omega,
                                                                      CgState *st, SweepSync *sy) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (stop_requested(&st->done)) return;
  // warps numbered across blocks first, as in csrv_sweep_kernel
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int wid = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
  const int total = sweep_passes(plan);
  bool zero = false;
  int c = -1;
  int q = sweep_next(plan, -1, total, c, zero);
  SellSlicePre<T, BT> pre;
  if (q < total) {
    const int s0 = plan.bounds[c], s1 = plan.bounds[c + 1];
    sell_slice_pre<T, BT, G>(A, b, s0 + wid, s0 + wid < s1, lane, pre);
  }
  unsigned barrier = 0;
  while (q < total) {
    const int s0 = plan.bounds[c], s1 = plan.bounds[c + 1];
    const int row_begin = plan.first_row[c];
    const T w = wts != nullptr ? wts[c] : omega;
    for (int s = s0 + wid; s < s1; s += warps) {  // uniform over the warp
      if (s != s0 + wid) sell_slice_pre<T, BT, G>(A, b, s, true, lane, pre);
      if (zero) sell_slice_update<T, BT, true, G>(A, pre, lane, x, w, row_begin);
      else sell_slice_update<T, BT, false, G>(A, pre, lane, x, w, row_begin);
    }
    int cn = -1;
    bool zn = false;
    const int qn = sweep_next(plan, q, total, cn, zn);
    if (qn < total) {
      const int n0 = plan.bounds[cn], n1 = plan.bounds[cn + 1];
      sell_slice_pre<T, BT, G>(A, b, n0 + wid, n0 + wid < n1, lane, pre);
      sweep_barrier(sy, st, ++barrier);
    }
    q = qn, c = cn, zero = zn;
  }
  sweep_leave(sy);
}

}  // namespace gsb
