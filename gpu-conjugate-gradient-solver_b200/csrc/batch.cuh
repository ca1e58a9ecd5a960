// Kernels of the batched AMG-PCG solver: many independent systems of uneven
// sizes, each with up to four right-hand sides, advanced together.
//
// Storage. Level k of the batch is the block-diagonal matrix of every
// system's level-k matrix, systems one after another, each system's rows in
// its own colour-contiguous order. The R right-hand sides of a system share
// its matrix: vectors are stored row-interleaved ([row][R]), so one read of a
// matrix entry serves R updates and a neighbour gather is one R-wide load.
//
// Work lists. Every launch walks a list of items (system, begin, end, aux):
// a range of SELL-32 slices or of rows of one system (never crossing systems
// or colours), with aux the first row of the item's colour where it matters.
// The blocks of a launch loop over the list (grid-stride), so one launch
// carries the same pass of every system: colour j of the forward sweep is
// colour j of each system, colour C_s - 1 - j of the backward sweep. An item
// whose system has finished (every right-hand side converged) is skipped.
//
// Outer CG (FP64). Per (system, right-hand side) pair the scalars live in
// BPair on the device. Item kernels write per-item partial sums; one block
// per system then adds its items' partials in a fixed order (deterministic)
// and updates the pair scalars and the convergence flags.
#pragma once

#include "kernels.cuh"

namespace gsb {

template <typename T, int R>
struct alignas(sizeof(T) * R) Rv {
  T v[R];
};

template <typename T, int R>
__device__ __forceinline__ Rv<T, R> rv_zero() {
  Rv<T, R> z;
#pragma unroll
  for (int j = 0; j < R; ++j) z.v[j] = T(0);
  return z;
}

// Read-only (non-coherent) load of the R values of one row.
template <typename T, int R>
__device__ __forceinline__ Rv<T, R> ldg_rv(const Rv<T, R> *p) {
  Rv<T, R> r;
  if constexpr (R == 4 && sizeof(T) == 4) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
    r.v[0] = q.x, r.v[1] = q.y, r.v[2] = q.z, r.v[3] = q.w;
  } else if constexpr (R == 4 && sizeof(T) == 8) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    r.v[0] = a.x, r.v[1] = a.y, r.v[2] = b.x, r.v[3] = b.y;
  } else {
#pragma unroll
    for (int j = 0; j < R; ++j) r.v[j] = __ldg(&p->v[j]);
  }
  return r;
}

template <typename T, int R>
__device__ __forceinline__ void fma_rv(T a, const Rv<T, R> &x, Rv<T, R> &acc) {
#pragma unroll
  for (int j = 0; j < R; ++j) acc.v[j] = fma(a, x.v[j], acc.v[j]);
}

// Items: x = system, y = begin, z = end, w = aux.
using BItem = int4;

__device__ __forceinline__ bool item_skipped(const int *sys_done, int sys) {
  return sys_done != nullptr && sys_done[sys] != 0;
}

// ---- SELL-32, one lane per row -------------------------------------------
template <typename T, int R, bool kSkip>
__device__ __forceinline__ Rv<T, R> bsell_offdiag(const SellView<T> &A, int s, int lane,
                                                  const Rv<T, R> *__restrict__ x, int skip_from) {
  using P2 = typename Pair<T>::type;
  const int p0 = A.sptr[s], p1 = A.sptr[s + 1];
  Rv<T, R> sum = rv_zero<T, R>();
#pragma unroll 2
  for (int p = p0 + 2 * lane; p < p1; p += 64) {
    const P2 v = __ldg(reinterpret_cast<const P2 *>(A.val + p));
    const int2 c = __ldg(reinterpret_cast<const int2 *>(A.col + p));
    if (!kSkip || c.x < skip_from) fma_rv<T, R>(v.x, ldg_rv<T, R>(x + c.x), sum);
    if (!kSkip || c.y < skip_from) fma_rv<T, R>(v.y, ldg_rv<T, R>(x + c.y), sum);
  }
  return sum;
}

// Gauss-Seidel colour pass, items = slice ranges of one colour of one system
// (aux = first row of that colour):
//     x_i <- (1 - w) x_i + w (b_i - sum_{j != i} a_ij x_j) / a_ii
// for each of the R right-hand sides. kZero: x is an implicit zero vector
// before this forward sweep (columns >= aux hold zero and are not read).
template <typename T, typename BT, int R, bool kZero>
__global__ void __launch_bounds__(256) bsell_gs_kernel(SellView<T> A, const BItem *__restrict__ items,
                                                       int nitems, const Rv<BT, R> *__restrict__ b,
                                                       Rv<T, R> *__restrict__ x, T w,
                                                       const int *__restrict__ sys_done) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    for (int s = q.y + warp; s < q.z; s += nw) {
      const Rv<T, R> off = bsell_offdiag<T, R, kZero>(A, s, lane, x, q.w);
      const int row = A.srow[s] + lane;
      if (row < A.srow[s + 1]) {
        const T d = A.diag[row];
        const Rv<BT, R> bv = b[row];
        Rv<T, R> xn;
        if (kZero) {
#pragma unroll
          for (int j = 0; j < R; ++j) xn.v[j] = w * ((T(bv.v[j]) - off.v[j]) / d);
        } else {
          const Rv<T, R> xo = x[row];
#pragma unroll
          for (int j = 0; j < R; ++j) xn.v[j] = (T(1) - w) * xo.v[j] + w * ((T(bv.v[j]) - off.v[j]) / d);
        }
        x[row] = xn;
      }
    }
  }
}

// y = A x (kSpmvSet), y = b - A x (kSpmvResid), y += A x (kSpmvAdd); items
// are slice ranges.
template <typename T, typename BT, int R, int kMode>
__global__ void __launch_bounds__(256) bsell_spmv_kernel(SellView<T> A, const BItem *__restrict__ items,
                                                         int nitems, const Rv<T, R> *__restrict__ x,
                                                         Rv<T, R> *__restrict__ y,
                                                         const Rv<BT, R> *__restrict__ b,
                                                         const int *__restrict__ sys_done) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    for (int s = q.y + warp; s < q.z; s += nw) {
      Rv<T, R> sum = bsell_offdiag<T, R, false>(A, s, lane, x, 0);
      const int row = A.srow[s] + lane;
      if (row < A.srow[s + 1]) {
        if (A.diag != nullptr) fma_rv<T, R>(A.diag[row], x[row], sum);
        Rv<T, R> out;
        if (kMode == kSpmvResid) {
          const Rv<BT, R> bv = b[row];
#pragma unroll
          for (int j = 0; j < R; ++j) out.v[j] = T(bv.v[j]) - sum.v[j];
        } else if (kMode == kSpmvAdd) {
          out = y[row];
#pragma unroll
          for (int j = 0; j < R; ++j) out.v[j] += sum.v[j];
        } else {
          out = sum;
        }
        y[row] = out;
      }
    }
  }
}

// ---- CSR-vector, G lanes per row -----------------------------------------
template <typename T, int R, bool kSkip, int G>
__device__ __forceinline__ Rv<T, R> bcsrv_offdiag(const CsrvView<T> &A, int row, bool valid, int sub,
                                                  const Rv<T, R> *__restrict__ x, int skip_from) {
  Rv<T, R> sum = rv_zero<T, R>();
  if (valid) {
    const int k1 = A.rp[row + 1];
#pragma unroll 4
    for (int k = A.rp[row] + sub; k < k1; k += G) {
      const int c = __ldg(A.ci + k);
      if (!kSkip || c < skip_from) fma_rv<T, R>(__ldg(A.v + k), ldg_rv<T, R>(x + c), sum);
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
    for (int j = 0; j < R; ++j) sum.v[j] += __shfl_xor_sync(0xffffffffu, sum.v[j], o, G);
  return sum;
}

// Items are row ranges of one colour of one system (aux = first row of the
// colour). Every lane of a block runs the same number of trips, so the
// shuffles see full warps.
template <typename T, typename BT, int R, bool kZero, int G>
__global__ void __launch_bounds__(256) bcsrv_gs_kernel(CsrvView<T> A, const BItem *__restrict__ items,
                                                       int nitems, const Rv<BT, R> *__restrict__ b,
                                                       Rv<T, R> *__restrict__ x, T w,
                                                       const int *__restrict__ sys_done) {
  const int sub = threadIdx.x & (G - 1), grp = threadIdx.x / G, ngrp = blockDim.x / G;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    const int trips = (q.z - q.y + ngrp - 1) / ngrp;
    for (int t = 0; t < trips; ++t) {
      const int row = q.y + grp + t * ngrp;
      const bool valid = row < q.z;
      const Rv<T, R> off = bcsrv_offdiag<T, R, kZero, G>(A, row, valid, sub, x, q.w);
      if (valid && sub == 0) {
        const T d = A.diag[row];
        const Rv<BT, R> bv = b[row];
        Rv<T, R> xn;
        if (kZero) {
#pragma unroll
          for (int j = 0; j < R; ++j) xn.v[j] = w * ((T(bv.v[j]) - off.v[j]) / d);
        } else {
          const Rv<T, R> xo = x[row];
#pragma unroll
          for (int j = 0; j < R; ++j) xn.v[j] = (T(1) - w) * xo.v[j] + w * ((T(bv.v[j]) - off.v[j]) / d);
        }
        x[row] = xn;
      }
    }
  }
}

template <typename T, typename BT, int R, int kMode, int G>
__global__ void __launch_bounds__(256) bcsrv_spmv_kernel(CsrvView<T> A, const BItem *__restrict__ items,
                                                         int nitems, const Rv<T, R> *__restrict__ x,
                                                         Rv<T, R> *__restrict__ y,
                                                         const Rv<BT, R> *__restrict__ b,
                                                         const int *__restrict__ sys_done) {
  const int sub = threadIdx.x & (G - 1), grp = threadIdx.x / G, ngrp = blockDim.x / G;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    const int trips = (q.z - q.y + ngrp - 1) / ngrp;
    for (int t = 0; t < trips; ++t) {
      const int row = q.y + grp + t * ngrp;
      const bool valid = row < q.z;
      Rv<T, R> sum = bcsrv_offdiag<T, R, false, G>(A, row, valid, sub, x, 0);
      if (valid && sub == 0) {
        if (A.diag != nullptr) fma_rv<T, R>(A.diag[row], x[row], sum);
        Rv<T, R> out;
        if (kMode == kSpmvResid) {
          const Rv<BT, R> bv = b[row];
#pragma unroll
          for (int j = 0; j < R; ++j) out.v[j] = T(bv.v[j]) - sum.v[j];
        } else if (kMode == kSpmvAdd) {
          out = y[row];
#pragma unroll
          for (int j = 0; j < R; ++j) out.v[j] += sum.v[j];
        } else {
          out = sum;
        }
        y[row] = out;
      }
    }
  }
}

// ---- coarsest levels: x_c = A_c^-1 b_c per system ---------------------------
// Items: x = system, y = its coarsest level, z/w = local row range. One warp
// per row of the system's dense FP64 inverse.
template <typename T, int R>
__global__ void __launch_bounds__(256) bdense_kernel(const BItem *__restrict__ items, int nitems,
                                                     const double *__restrict__ ainv,
                                                     const long long *__restrict__ ainv_off,
                                                     const int *__restrict__ crow0,
                                                     const int *__restrict__ cn,
                                                     Rv<T, R> *const *__restrict__ xl,
                                                     const Rv<T, R> *const *__restrict__ bl,
                                                     const int *__restrict__ sys_done) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    const int n = cn[q.x], r0 = crow0[q.x];
    const Rv<T, R> *b = bl[q.y] + r0;
    Rv<T, R> *x = xl[q.y] + r0;
    const double *a = ainv + ainv_off[q.x];
    for (int row = q.z + warp; row < q.w; row += nw) {
      const double *ar = a + static_cast<size_t>(row) * n;
      double acc[R];
#pragma unroll
      for (int j = 0; j < R; ++j) acc[j] = 0.0;
      for (int c = lane; c < n; c += 32) {
        const double av = __ldg(ar + c);
        const Rv<T, R> bv = ldg_rv<T, R>(b + c);
#pragma unroll
        for (int j = 0; j < R; ++j) acc[j] = fma(av, double(bv.v[j]), acc[j]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
      if (lane == 0) {
        Rv<T, R> out;
#pragma unroll
        for (int j = 0; j < R; ++j) out.v[j] = T(acc[j]);
        x[row] = out;
      }
    }
  }
}

// ---- outer CG (FP64) ------------------------------------------------------
// Scalars of one (system, right-hand side) pair.
struct BPair {
  double rho, alpha, beta, rr, bb, ratio, pAp;
  int iter, done, status, iterations;
};

struct BCgShared {
  double tol2;
  int max_iter;
  int flexible;
  int active;  // systems with at least one pair still running (after the last convergence test)
};

// Deterministic block sum of kN values per thread into smem-backed totals;
// the result is valid in thread 0.
template <int kN>
__device__ __forceinline__ void bblock_sum(double (&v)[kN], double *smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < kN; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < kN; ++i) smem[warp * kN + i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < kN; ++i) {
      double t = 0.0;
      for (int q = 0; q < nw; ++q) t += smem[q * kN + i];
      v[i] = t;
    }
  }
}

// CG items: x = system, y/z = slice range of level 0, w unused. Rows are
// [srow[y], srow[z]).

// Ap = A p and the per-item partials of p . Ap (R values per item).
template <int R>
__global__ void __launch_bounds__(256) bcg_spmv_pap_kernel(SellView<double> A, const BItem *__restrict__ items,
                                                           int nitems, const Rv<double, R> *__restrict__ p,
                                                           Rv<double, R> *__restrict__ ap,
                                                           const int *__restrict__ sys_done,
                                                           double *__restrict__ partials) {
  __shared__ double smem[32 * R];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) acc[j] = 0.0;
    for (int s = q.y + warp; s < q.z; s += nw) {
      Rv<double, R> sum = bsell_offdiag<double, R, false>(A, s, lane, p, 0);
      const int row = A.srow[s] + lane;
      if (row < A.srow[s + 1]) {
        const Rv<double, R> pr = p[row];
        fma_rv<double, R>(A.diag[row], pr, sum);
        ap[row] = sum;
#pragma unroll
        for (int j = 0; j < R; ++j) acc[j] = fma(pr.v[j], sum.v[j], acc[j]);
      }
    }
    bblock_sum<R>(acc, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int j = 0; j < R; ++j) partials[static_cast<size_t>(it) * R + j] = acc[j];
  }
}

// x += alpha p, r -= alpha Ap for running pairs; partials of r . r.
template <int R>
__global__ void __launch_bounds__(256) bcg_update_xr_kernel(const int *__restrict__ srow,
                                                            const BItem *__restrict__ items, int nitems,
                                                            Rv<double, R> *__restrict__ x,
                                                            Rv<double, R> *__restrict__ r,
                                                            const Rv<double, R> *__restrict__ p,
                                                            const Rv<double, R> *__restrict__ ap,
                                                            const BPair *__restrict__ pairs,
                                                            const int *__restrict__ sys_done,
                                                            double *__restrict__ partials) {
  __shared__ double smem[32 * R];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    double alpha[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const BPair &pr = pairs[q.x * R + j];
      alpha[j] = pr.done ? 0.0 : pr.alpha;
    }
    double acc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) acc[j] = 0.0;
    const int r1 = srow[q.z];
    for (int i = srow[q.y] + threadIdx.x; i < r1; i += blockDim.x) {
      Rv<double, R> xi = x[i], ri = r[i];
      const Rv<double, R> pi = p[i], api = ap[i];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (alpha[j] != 0.0) {
          xi.v[j] = fma(alpha[j], pi.v[j], xi.v[j]);
          ri.v[j] = fma(-alpha[j], api.v[j], ri.v[j]);
        }
        acc[j] = fma(ri.v[j], ri.v[j], acc[j]);
      }
      x[i] = xi;
      r[i] = ri;
    }
    bblock_sum<R>(acc, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int j = 0; j < R; ++j) partials[static_cast<size_t>(it) * R + j] = acc[j];
  }
}

// Partials of r . z and (flexible) r . z_old: 2R values per item.
template <typename ZT, int R>
__global__ void __launch_bounds__(256) bcg_dot_rz_kernel(const int *__restrict__ srow,
                                                         const BItem *__restrict__ items, int nitems,
                                                         const Rv<double, R> *__restrict__ r,
                                                         const Rv<ZT, R> *__restrict__ z,
                                                         const Rv<ZT, R> *__restrict__ z_old,
                                                         const int *__restrict__ sys_done,
                                                         double *__restrict__ partials) {
  __shared__ double smem[32 * 2 * R];
  const bool flex = z_old != nullptr;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    double acc[2 * R];
#pragma unroll
    for (int j = 0; j < 2 * R; ++j) acc[j] = 0.0;
    const int r1 = srow[q.z];
    for (int i = srow[q.y] + threadIdx.x; i < r1; i += blockDim.x) {
      const Rv<double, R> ri = r[i];
      const Rv<ZT, R> zi = z[i];
#pragma unroll
      for (int j = 0; j < R; ++j) acc[j] = fma(ri.v[j], double(zi.v[j]), acc[j]);
      if (flex) {
        const Rv<ZT, R> zo = z_old[i];
#pragma unroll
        for (int j = 0; j < R; ++j) acc[R + j] = fma(ri.v[j], double(zo.v[j]), acc[R + j]);
      }
    }
    bblock_sum<2 * R>(acc, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int j = 0; j < 2 * R; ++j) partials[static_cast<size_t>(it) * 2 * R + j] = acc[j];
  }
}

// p = z + beta p for running pairs.
template <typename ZT, int R>
__global__ void __launch_bounds__(256) bcg_update_p_kernel(const int *__restrict__ srow,
                                                           const BItem *__restrict__ items, int nitems,
                                                           const Rv<ZT, R> *__restrict__ z,
                                                           Rv<double, R> *__restrict__ p,
                                                           const BPair *__restrict__ pairs,
                                                           const int *__restrict__ sys_done) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    if (item_skipped(sys_done, q.x)) continue;
    double beta[R];
    bool run[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const BPair &pr = pairs[q.x * R + j];
      run[j] = pr.done == 0;
      beta[j] = pr.beta;
    }
    const int r1 = srow[q.z];
    for (int i = srow[q.y] + threadIdx.x; i < r1; i += blockDim.x) {
      const Rv<ZT, R> zi = z[i];
      Rv<double, R> pi = p[i];
#pragma unroll
      for (int j = 0; j < R; ++j)
        if (run[j]) pi.v[j] = fma(beta[j], pi.v[j], double(zi.v[j]));
      p[i] = pi;
    }
  }
}

// Start of the solve: p = z; partials of b . b, r . z, r . r (3R per item).
template <typename ZT, int R>
__global__ void __launch_bounds__(256) bcg_init_kernel(const int *__restrict__ srow,
                                                       const BItem *__restrict__ items, int nitems,
                                                       const Rv<double, R> *__restrict__ b,
                                                       const Rv<double, R> *__restrict__ r,
                                                       const Rv<ZT, R> *__restrict__ z,
                                                       Rv<double, R> *__restrict__ p,
                                                       double *__restrict__ partials) {
  __shared__ double smem[32 * 3 * R];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BItem q = items[it];
    double acc[3 * R];
#pragma unroll
    for (int j = 0; j < 3 * R; ++j) acc[j] = 0.0;
    const int r1 = srow[q.z];
    for (int i = srow[q.y] + threadIdx.x; i < r1; i += blockDim.x) {
      const Rv<double, R> bi = b[i], ri = r[i];
      const Rv<ZT, R> zi = z[i];
      Rv<double, R> pi;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const double zj = double(zi.v[j]);
        pi.v[j] = zj;
        acc[j] = fma(bi.v[j], bi.v[j], acc[j]);
        acc[R + j] = fma(ri.v[j], zj, acc[R + j]);
        acc[2 * R + j] = fma(ri.v[j], ri.v[j], acc[2 * R + j]);
      }
      p[i] = pi;
    }
    bblock_sum<3 * R>(acc, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int j = 0; j < 3 * R; ++j) partials[static_cast<size_t>(it) * 3 * R + j] = acc[j];
  }
}

// Sum of one system's item partials (stride kN per item, component i), in a
// fixed order: lane-strided over the items, then a fixed shuffle tree.
template <int kN>
__device__ __forceinline__ double sum_items(const double *partials, int i0, int i1, int comp, int lane) {
  double t = 0.0;
  for (int i = i0 + lane; i < i1; i += 32) t += partials[static_cast<size_t>(i) * kN + comp];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

// Finalize kernels: one block of 32*R threads per system, warp j handles the
// pair (system, j).
enum BFinal : int { kBFinInit = 0, kBFinPap = 1, kBFinXr = 2, kBFinRz = 3 };

template <int R, int kWhich>
__global__ void __launch_bounds__(128) bcg_finalize_kernel(const int *__restrict__ item_first,
                                                           const double *__restrict__ partials,
                                                           BPair *__restrict__ pairs, int *__restrict__ sys_done,
                                                           BCgShared *__restrict__ sh) {
  const int s = blockIdx.x, j = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (kWhich == kBFinPap && s == 0 && threadIdx.x == 0) sh->active = 0;
  __shared__ int any_running;
  if (threadIdx.x == 0) any_running = 0;
  __syncthreads();
  const bool skip = kWhich != kBFinInit && sys_done[s] != 0;
  if (!skip) {
    const int i0 = item_first[s], i1 = item_first[s + 1];
    BPair &P = pairs[s * R + j];
    if (kWhich == kBFinInit) {
      const double bb = sum_items<3 * R>(partials, i0, i1, j, lane);
      const double rz = sum_items<3 * R>(partials, i0, i1, R + j, lane);
      const double rr = sum_items<3 * R>(partials, i0, i1, 2 * R + j, lane);
      if (lane == 0) {
        P.bb = bb;
        P.rho = rz;
        P.rr = rr;
        P.ratio = rr / bb;
        P.iter = 0;
        P.iterations = 0;
        P.alpha = P.beta = P.pAp = 0.0;
        P.done = 0;
        P.status = kCgRunning;
        if (!(sqrt(bb) >= 1e-12)) {
          // CGSolver::solve: a zero right-hand side returns x = 0
          P.status = isfinite(bb) ? kCgZeroRhs : kCgNotFinite;
          P.done = 1;
        } else if (!isfinite(P.ratio)) {
          P.status = kCgNotFinite;
          P.done = 1;
        } else if (P.ratio < sh->tol2) {
          P.status = kCgInitialConverged;
          P.done = 1;
        }
        if (!P.done) atomicOr(&any_running, 1);
      }
    } else if (kWhich == kBFinPap) {
      const double pap = sum_items<R>(partials, i0, i1, j, lane);
      if (lane == 0 && !P.done) {
        P.pAp = pap;
        if (!isfinite(pap) || pap == 0.0) {
          P.status = pap == 0.0 ? kCgBreakdown : kCgNotFinite;
          P.done = 1;
          P.iterations = P.iter;
          P.alpha = 0.0;
        } else {
          P.alpha = P.rho / pap;
        }
      }
    } else if (kWhich == kBFinXr) {
      const double rr = sum_items<R>(partials, i0, i1, j, lane);
      if (lane == 0 && !P.done) {
        P.rr = rr;
        const double ratio = rr / P.bb;
        P.ratio = ratio;
        if (!isfinite(ratio)) {
          P.status = kCgNotFinite;
          P.done = 1;
          P.iterations = P.iter;
        } else if (ratio < sh->tol2) {
          P.status = kCgConverged;
          P.done = 1;
          P.iterations = P.iter;  // 0-based, as the reference counts
        } else if (P.iter + 1 >= sh->max_iter) {
          P.status = kCgMaxIter;
          P.done = 1;
          P.iterations = sh->max_iter;
        }
        P.iter += 1;
      }
      if (lane == 0 && !P.done) atomicOr(&any_running, 1);
    } else {  // kBFinRz
      const double rz = sum_items<2 * R>(partials, i0, i1, j, lane);
      const double rzo = sum_items<2 * R>(partials, i0, i1, R + j, lane);
      if (lane == 0 && !P.done) {
        P.beta = (sh->flexible ? (rz - rzo) : rz) / P.rho;
        P.rho = rz;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && (kWhich == kBFinInit || kWhich == kBFinXr) && !skip) {
    sys_done[s] = any_running ? 0 : 1;
    if (any_running) atomicAdd(&sh->active, 1);
  }
}

// ---- caller layout <-> internal layout ------------------------------------
// Caller: system s occupies [uoff[s], uoff[s] + nrhs * n[s]), right-hand side
// j of s at uoff[s] + j * n[s], rows in the caller's order. Internal: row
// q0[qoff[s] + i] + off0[s] of level 0, R values per row; columns j >= nrhs
// are set to zero. blockIdx.y = system.
template <int R>
__global__ void bscatter_kernel(const long long *__restrict__ uoff, const int *__restrict__ n,
                                const int *__restrict__ off0, const long long *__restrict__ qoff,
                                const int *__restrict__ q0, int nrhs, const double *__restrict__ in,
                                Rv<double, R> *__restrict__ out) {
  const int s = blockIdx.y, ns = n[s];
  const double *src = in + uoff[s];
  const int *q = q0 + qoff[s];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    Rv<double, R> v;
#pragma unroll
    for (int j = 0; j < R; ++j) v.v[j] = j < nrhs ? src[static_cast<size_t>(j) * ns + i] : 0.0;
    out[off0[s] + q[i]] = v;
  }
}

// Inverse of bscatter_kernel; pairs that ended with a zero right-hand side
// return x = 0.
template <int R>
__global__ void bgather_kernel(const long long *__restrict__ uoff, const int *__restrict__ n,
                               const int *__restrict__ off0, const long long *__restrict__ qoff,
                               const int *__restrict__ q0, int nrhs, const Rv<double, R> *__restrict__ in,
                               const BPair *__restrict__ pairs, double *__restrict__ out) {
  const int s = blockIdx.y, ns = n[s];
  double *dst = out + uoff[s];
  const int *q = q0 + qoff[s];
  bool zero[R];
#pragma unroll
  for (int j = 0; j < R; ++j) zero[j] = pairs[s * R + j].status == kCgZeroRhs;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const Rv<double, R> v = in[off0[s] + q[i]];
#pragma unroll
    for (int j = 0; j < R; ++j)
      if (j < nrhs) dst[static_cast<size_t>(j) * ns + i] = zero[j] ? 0.0 : v.v[j];
  }
}

}  // namespace gsb
