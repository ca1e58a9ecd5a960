// Device kernels of the AMG-PCG hot path (sm_100a). Every kernel here is
// bandwidth-bound: none uses tensor cores.
//
// Matrix layout, "SELL-32": rows are cut into slices of at most 32
// consecutive rows (one warp, one row per lane). A slice never crosses a
// colour boundary, so a Gauss-Seidel colour pass is a contiguous range of
// slices. Inside a slice the off-diagonal entries are stored slot-pair
// interleaved: entry (slot k, lane l) of slice s sits at
//     sptr[s] + (k / 2) * 64 + 2 * l + (k % 2),
// so each lane loads two values (one 128-bit load in FP64) and two column
// indices (one 64-bit load) per step and a warp's loads are contiguous. The
// slice width (sptr[s+1]-sptr[s])/32 is even; padding entries carry value 0
// and a column inside the slice's own rows. The diagonal of a square level
// matrix is held apart in diag[] (it is the Gauss-Seidel divisor).
//
// The 3x3 block variant ("BELL-32") holds one block row (node) per lane;
// block slot q, component c (row-major 3x3) of lane l of slice s is at
//     9 * bptr[s] + (q * 9 + c) * 32 + l,   block column at bptr[s] + q*32 + l,
// with the diagonal blocks and their inverses apart (9 per node, row-major).
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace gsb {

template <typename T>
struct SellView {
  int rows, cols, nslices;
  const int *__restrict__ srow;  // nslices + 1: first row of each slice
  const int *__restrict__ sptr;  // nslices + 1: element offset of each slice
  const int *__restrict__ col;
  const T *__restrict__ val;
  const T *__restrict__ diag;    // rows, or nullptr (transfer operators)
};

template <typename T>
struct BellView {
  int nodes, nslices;
  const int *__restrict__ srow;  // nslices + 1: first node of each slice
  const int *__restrict__ bptr;  // nslices + 1: block-slot offset of each slice
  const int *__restrict__ col;   // block column per block slot
  const T *__restrict__ val;     // 9 per block slot, component-major per slice
  const T *__restrict__ diag;    // 9 per node
  const T *__restrict__ dinv;    // 9 per node
};

// State of one preconditioned CG solve, resident on the device. Scalars are
// produced by the last block of each reduction kernel; the host reads
// `done`/`status` only when it has to.
struct CgState {
  double rho, rho_new, rz_old, pAp, alpha, beta, rr, bb, ratio, tol2;
  int iter, max_iter, done, status, iterations, flexible;
  unsigned int ticket;
  int sync_fault;  // a bounded grid-barrier wait gave up (cooperative sweeps)
};

enum CgStatus : int {
  kCgRunning = 0,
  kCgConverged = 1,
  kCgMaxIter = 2,
  kCgNotFinite = 3,
  kCgBreakdown = 4,
  kCgInitialConverged = 5,
  kCgZeroRhs = 6,
};

// kSpmvTwice writes y = (A x) + (A x): the reference's prolongation on a
// level below the finest, whose correction buffer is the solution itself.
enum SpmvMode : int { kSpmvSet = 0, kSpmvResid = 1, kSpmvAdd = 2, kSpmvTwice = 3 };

template <typename T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

__device__ __forceinline__ bool stop_requested(const int *done) {
  return done != nullptr && *reinterpret_cast<const volatile int *>(done) != 0;
}

// Entry of every V-cycle kernel. Launched with programmatic stream
// serialization, a kernel's CTAs may become resident while its predecessor in
// the stream is still draining: griddepcontrol.wait holds them until that
// predecessor has completed and its writes are visible, and only then does the
// kernel let its own successor start launching. Every thread waits before its
// first memory access (the stop flag included) and before any early return,
// so completion of this grid still implies completion of all earlier work.
// Without the launch attribute both instructions are no-ops.
__device__ __forceinline__ bool pass_entry(const int *done) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  return stop_requested(done);
}

// Off-diagonal row sum of lane `lane` of slice s: sum_k val * x[col].
// With kSkipFrom >= 0 (zero initial guess, first forward sweep), columns at
// or above `skip_from` are known to hold zero and are not gathered.
template <typename T, bool kSkip>
__device__ __forceinline__ T sell_offdiag(const SellView<T> &A, int s, int lane,
                                          const T *__restrict__ x, int skip_from) {
  using P2 = typename Pair<T>::type;
  const int p0 = A.sptr[s], p1 = A.sptr[s + 1];
  T sum = T(0);
#pragma unroll 4
  for (int p = p0 + 2 * lane; p < p1; p += 64) {
    const P2 v = __ldg(reinterpret_cast<const P2 *>(A.val + p));
    const int2 c = __ldg(reinterpret_cast<const int2 *>(A.col + p));
    if (kSkip) {
      if (c.x < skip_from) sum = fma(v.x, __ldg(x + c.x), sum);
      if (c.y < skip_from) sum = fma(v.y, __ldg(x + c.y), sum);
    } else {
      sum = fma(v.x, __ldg(x + c.x), sum);
      sum = fma(v.y, __ldg(x + c.y), sum);
    }
  }
  return sum;
}

// Operands of one slice that do not depend on the iterate: its row range and
// each lane's first kPairs slot pairs.
template <typename T>
struct SellHead {
  static constexpr int kPairs = 2;  // slot pairs held per lane (FP32 fits 32 registers)
  int r0, r1, p0, p1;
  typename Pair<T>::type v[kPairs];
  int2 c[kPairs];
};

// Loads the head of slice s (bounds and the lane's first slot pairs).
template <typename T>
__device__ __forceinline__ void sell_head_ops(const SellView<T> &A, int s, int lane, SellHead<T> &h) {
  using P2 = typename Pair<T>::type;
  h.r0 = __ldg(A.srow + s);
  h.r1 = __ldg(A.srow + s + 1);
  h.p0 = __ldg(A.sptr + s);
  h.p1 = __ldg(A.sptr + s + 1);
#pragma unroll
  for (int q = 0; q < SellHead<T>::kPairs; ++q) {
    const int p = h.p0 + 2 * lane + 64 * q;
    if (p < h.p1) {
      h.v[q] = __ldg(reinterpret_cast<const P2 *>(A.val + p));
      h.c[q] = __ldg(reinterpret_cast<const int2 *>(A.col + p));
    } else {
      h.v[q].x = h.v[q].y = T(0);
      h.c[q] = make_int2(-1, -1);
    }
  }
}

// Loads the head of slice s; returns the diagonal of the lane's row (1 for
// lanes that hold no row start).
template <typename T, int G>
__device__ __forceinline__ T sell_head(const SellView<T> &A, int s, int lane, SellHead<T> &h) {
  sell_head_ops(A, s, lane, h);
  const int row = h.r0 + lane / G;
  return ((lane & (G - 1)) == 0 && row < h.r1) ? __ldg(A.diag + row) : T(1);
}

// The lane's off-diagonal sum from a loaded head. The pair after the head is
// loaded first (it overlaps the head's gathers), then the slots past it for
// wider slices. Same summation order as sell_offdiag.
// Neighbour value for a colour pass: column c from the iterate, or, when
// `xp` is given (a colouring that lets weakly coupled rows share a colour),
// from the iterate the sweep started with for the columns of the pass's own
// colour [lo, hi) (Jacobi within the colour: no row of the pass reads a value
// another row of the same pass writes).
// kRel false: the plain load (the exact colourings' passes carry no select,
// which would cost registers in kernels held to 32 or 128).
template <bool kRel, typename T>
__device__ __forceinline__ T nb_load(const T *__restrict__ x, const T *__restrict__ xp, int lo, int hi, int c) {
  if constexpr (kRel) return __ldg((c >= lo && c < hi ? xp : x) + c);
  else return __ldg(x + c);
}

template <typename T, bool kSkip, bool kRel = false>
__device__ __forceinline__ T sell_offdiag_head(const SellView<T> &A, const SellHead<T> &h, int lane,
                                               const T *__restrict__ x, int skip_from,
                                               const T *__restrict__ xp = nullptr, int lo = 0, int hi = 0) {
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
    g[2 * q] = ok0 ? nb_load<kRel>(x, xp, lo, hi, h.c[q].x) : T(0);
    g[2 * q + 1] = ok1 ? nb_load<kRel>(x, xp, lo, hi, h.c[q].y) : T(0);
  }
  {
    const bool ok0 = cn.x >= 0 && (!kSkip || cn.x < skip_from);
    const bool ok1 = cn.y >= 0 && (!kSkip || cn.y < skip_from);
    g[2 * kP] = ok0 ? nb_load<kRel>(x, xp, lo, hi, cn.x) : T(0);
    g[2 * kP + 1] = ok1 ? nb_load<kRel>(x, xp, lo, hi, cn.y) : T(0);
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
    if (!kSkip || c.x < skip_from) sum = fma(v.x, nb_load<kRel>(x, xp, lo, hi, c.x), sum);
    if (!kSkip || c.y < skip_from) sum = fma(v.y, nb_load<kRel>(x, xp, lo, hi, c.y), sum);
  }
  return sum;
}

// y = A x (kSpmvSet), y = b - A x (kSpmvResid), y += A x (kSpmvAdd).
// One warp per slice, grid-stride over slices. G lanes per row: a slice holds
// 32 / G rows, lane l serves row l / G and the group adds its partial sums.
template <typename T, typename BT, int kMode, int G = 1>
__global__ void __launch_bounds__(256) sell_spmv_kernel(SellView<T> A, const T *__restrict__ x,
                                                        T *__restrict__ y,
                                                        const BT *__restrict__ b,
                                                        const int *done) {
  if (pass_entry(done)) return;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  // Bandwidth-bound on the big levels: no head held across trips (it costs
  // occupancy, measured slower on the fine-level residual and prolongation)
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslices; s += warps) {
    T sum = sell_offdiag<T, false>(A, s, lane, x, 0);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const int row = A.srow[s] + lane / G;
    if ((lane & (G - 1)) == 0 && row < A.srow[s + 1]) {
      if (A.diag != nullptr) sum = fma(A.diag[row], x[row], sum);
      if (kMode == kSpmvSet) y[row] = sum;
      else if (kMode == kSpmvResid) y[row] = T(b[row]) - sum;
      else if (kMode == kSpmvTwice) y[row] = sum + sum;
      else y[row] += sum;
    }
  }
}

// One multicolour Gauss-Seidel pass over the slices [s_begin, s_end) of one
// colour (rows [row_begin, ...)), in place on x:
//     x_i <- (1 - w) x_i + w (b_i - sum_{j != i} a_ij x_j) / a_ii.
// kZero: x is an implicit zero vector before this forward sweep, so x_i and
// every neighbour in this or a later colour (column >= row_begin) count as 0.
// FP32: 8 resident blocks per SM (<= 32 registers, no spills), so the grid
// (8 blocks per SM, grid-stride over slices) is exactly one wave. FP64 needs
// more registers; its grid follows the occupancy the runtime reports.
template <typename T, typename BT, bool kZero, int G = 1, bool kRel = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 1) sell_gs_kernel(SellView<T> A, int s_begin, int s_end,
                                                      int row_begin, const BT *__restrict__ b,
                                                      T *__restrict__ x, const T *__restrict__ wts,
                                                      T omega, const int *done,
                                                      const T *__restrict__ xprev = nullptr, int row_end = 0) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int first = s_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  // The first slice's matrix operands and diagonal do not change during a
  // solve: they are loaded before the pass waits on its predecessor, so under
  // programmatic dependent launch they arrive while that pass drains.
  SellHead<T> h;
  T di = T(1);
  if (first < s_end) di = sell_head<T, G>(A, first, lane, h);
  if (pass_entry(done)) return;
  const T w = wts != nullptr ? wts[0] : omega;
  // grid-stride over the colour's slices: resident warps stay busy instead
  // of the grid running in partial waves
  for (int s = first; s < s_end; s += warps) {
    if (s != first) di = sell_head<T, G>(A, s, lane, h);
    // the row's own operands do not depend on the neighbour sum: issue their
    // loads first so they overlap the gathers
    const int row = h.r0 + lane / G;
    const bool valid = (lane & (G - 1)) == 0 && row < h.r1;
    T bi = T(0), xi = T(0);
    if (valid) {
      bi = T(__ldg(b + row));
      if (!kZero) xi = x[row];
    }
    T off = sell_offdiag_head<T, kZero, kRel>(A, h, lane, x, row_begin, xprev, row_begin, row_end);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
    if (valid) {
      const T gs = (bi - off) / di;
      x[row] = kZero ? w * gs : (T(1) - w) * xi + w * gs;
    }
  }
}

// ---- CSR-vector kernels: G lanes per row --------------------------------------
// For levels whose rows are long (Galerkin coarse operators carry 30-90
// entries per row) and whose colours hold few rows, one lane per row leaves
// each pass a long serial chain of loads. Here G consecutive lanes share a
// row: lane j of the group reads entries rp[row] + j, + j + G, ... (adjacent
// lanes read adjacent entries) and the group reduces with shuffles. The
// diagonal is held apart as in SELL-32; rows of one colour are contiguous.
template <typename T>
struct CsrvView {
  int rows;
  const int *__restrict__ rp;
  const int *__restrict__ ci;
  const T *__restrict__ v;
  const T *__restrict__ diag;  // rows, or nullptr
};

template <typename T, bool kSkip, int G>
__device__ __forceinline__ T csrv_offdiag(const CsrvView<T> &A, int row, bool valid, int sub,
                                          const T *__restrict__ x, int skip_from) {
  T sum = T(0);
  if (valid) {
    const int k1 = A.rp[row + 1];
    // chunks of 4 entries per lane: the 4 column loads, then their 4 gathers
    // and values, then the FMAs, so a chunk costs two dependent round trips
    for (int k0 = A.rp[row] + sub; k0 < k1; k0 += 4 * G) {
      int c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = k0 + u * G < k1 ? __ldg(A.ci + k0 + u * G) : -1;
      T xv[4], v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool use = c[u] >= 0 && (!kSkip || c[u] < skip_from);
        xv[u] = use ? __ldg(x + c[u]) : T(0);
        v[u] = c[u] >= 0 ? __ldg(A.v + k0 + u * G) : T(0);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) sum = fma(v[u], xv[u], sum);
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
  return sum;
}

// Operands of a row's first kE entries per lane that do not depend on the
// iterate. The size changes only how many entries are loaded before the wait
// on the predecessor: every lane still sums its entries in increasing order
// with one FMA chain, so the sums are the same bits for every kE.
template <typename T, int kE = 8>
struct CsrvHead {
  static constexpr int kEntries = kE;
  int k0, k1;
  int c[kEntries];
  T v[kEntries];
};

template <typename T, int G, int kE>
__device__ __forceinline__ void csrv_head(const CsrvView<T> &A, int row, bool valid, int sub, CsrvHead<T, kE> &h) {
  h.k0 = 0;
  h.k1 = 0;
  if (valid) {
    h.k0 = __ldg(A.rp + row) + sub;
    h.k1 = __ldg(A.rp + row + 1);
  }
#pragma unroll
  for (int u = 0; u < kE; ++u) {
    const int k = h.k0 + u * G;
    const bool in = k < h.k1;
    h.c[u] = in ? __ldg(A.ci + k) : -1;
    h.v[u] = in ? __ldg(A.v + k) : T(0);
  }
}

// csrv_offdiag from a loaded head: the same chunks in the same order.
template <typename T, bool kSkip, int G, int kE, bool kRel = false>
__device__ __forceinline__ T csrv_offdiag_head(const CsrvView<T> &A, const CsrvHead<T, kE> &h, int sub,
                                               const T *__restrict__ x, int skip_from,
                                               const T *__restrict__ xp = nullptr, int lo = 0, int hi = 0) {
  T sum = T(0);
  {
    T xv[kE];
#pragma unroll
    for (int u = 0; u < kE; ++u) {
      const bool use = h.c[u] >= 0 && (!kSkip || h.c[u] < skip_from);
      xv[u] = use ? nb_load<kRel>(x, xp, lo, hi, h.c[u]) : T(0);
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
      xv[u] = use ? nb_load<kRel>(x, xp, lo, hi, c[u]) : T(0);
      v[u] = c[u] >= 0 ? __ldg(A.v + k0 + u * G) : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) sum = fma(v[u], xv[u], sum);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, G);
  return sum;
}

template <typename T, typename BT, int kMode, int G>
__global__ void __launch_bounds__(256) csrv_spmv_kernel(CsrvView<T> A, const T *__restrict__ x,
                                                        T *__restrict__ y,
                                                        const BT *__restrict__ b,
                                                        const int *done) {
  const int sub = threadIdx.x & (G - 1);
  const int groups = (gridDim.x * blockDim.x) / G;
  // every lane of a warp runs the same number of trips so the shuffles
  // inside csrv_offdiag_head see full warps
  const int first = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int trips = (A.rows + groups - 1) / groups;
  // The first row's head (64 entries per row from 8 lanes up) is loaded
  // before the wait on the predecessor, and every trip loads the next row's
  // while its own gathers are in flight. Same sums as csrv_offdiag.
  CsrvHead<T, (G >= 8 ? 8 : 64 / G)> h;
  csrv_head<T, G>(A, first, first < A.rows, sub, h);
  if (pass_entry(done)) return;
  for (int t = 0; t < trips; ++t) {
    const int row = first + t * groups;
    const bool valid = row < A.rows;
    CsrvHead<T, (G >= 8 ? 8 : 64 / G)> hn;
    const bool more = t + 1 < trips;
    if (more) csrv_head<T, G>(A, row + groups, row + groups < A.rows, sub, hn);
    T sum = csrv_offdiag_head<T, false, G>(A, h, sub, x, 0);
    if (more) h = hn;
    if (valid && sub == 0) {
      if (A.diag != nullptr) sum = fma(A.diag[row], x[row], sum);
      if (kMode == kSpmvSet) y[row] = sum;
      else if (kMode == kSpmvResid) y[row] = T(b[row]) - sum;
      else if (kMode == kSpmvTwice) y[row] = sum + sum;
      else y[row] += sum;
    }
  }
}

template <typename T, typename BT, bool kZero, int G, bool kRel = false>
__global__ void __launch_bounds__(256) csrv_gs_kernel(CsrvView<T> A, int row_begin, int row_end,
                                                      const BT *__restrict__ b, T *__restrict__ x,
                                                      const T *__restrict__ wts, T omega,
                                                      const int *done, const T *__restrict__ xprev = nullptr) {
  const int sub = threadIdx.x & (G - 1);
  const int row = row_begin + (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = row < row_end;
  // matrix operands first (constant during a solve), then the wait on the
  // predecessor pass, then the iterate; 64 entries per row (8 per lane from
  // 8 lanes up), enough for the Galerkin rows of the coarse levels
  CsrvHead<T, (G >= 8 ? 8 : 64 / G)> h;
  csrv_head<T, G>(A, row, valid, sub, h);
  const T di = valid && sub == 0 ? __ldg(A.diag + row) : T(1);
  if (pass_entry(done)) return;
  const T off = csrv_offdiag_head<T, kZero, G, (G >= 8 ? 8 : 64 / G), kRel>(A, h, sub, x, row_begin, xprev, row_begin,
                                                                          row_end);
  if (valid && sub == 0) {
    const T w = wts != nullptr ? wts[0] : omega;
    const T gs = (T(b[row]) - off) / di;
    x[row] = kZero ? w * gs : (T(1) - w) * x[row] + w * gs;
  }
}

// ---- 3x3 block kernels ----------------------------------------------------
template <typename T, bool kSkip>
__device__ __forceinline__ void bell_offdiag(const BellView<T> &A, int s, int lane,
                                             const T *__restrict__ x, int skip_from, T acc[3]) {
  const int q0 = A.bptr[s], q1 = A.bptr[s + 1];
  acc[0] = acc[1] = acc[2] = T(0);
  // kSlots block slots per step: all column loads, then all gathers and value
  // loads, then the FMAs in slot order (the same sums as one slot at a time)
  // 8 slots in FP32 (128 registers), 4 in FP64 (about 120), no spills; fewer
  // measured slower on E64 (fine-level sweep 0.37 -> 0.51 of HBM peak)
  constexpr int kSlots = sizeof(T) == 4 ? 8 : 4;
  for (int q = q0; q < q1; q += 32 * kSlots) {
    // The slot bound is known before any column arrives, so the block values
    // are requested together with the columns (padding slots inside a slice
    // hold zero blocks and a valid column); only the gathers wait on them.
    int bc[kSlots];
    bool in[kSlots], use[kSlots];
    T xv[kSlots][3], vv[kSlots][9];
    const T *va = A.val + 9 * static_cast<size_t>(q) + lane;
#pragma unroll
    for (int u = 0; u < kSlots; ++u) {
      in[u] = q + 32 * u < q1;  // uniform over the warp
      bc[u] = in[u] ? __ldg(A.col + q + 32 * u + lane) : -1;
#pragma unroll
      for (int e = 0; e < 9; ++e) vv[u][e] = in[u] ? __ldg(va + (9 * u + e) * 32) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u) {
      use[u] = in[u] && (!kSkip || bc[u] < skip_from);
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[u][c] = use[u] ? __ldg(x + 3 * bc[u] + c) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u)
      if (use[u])
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[r] = fma(vv[u][3 * r + c], xv[u][c], acc[r]);
  }
}

// The first kSlots block slots of a lane of slice s (block columns and
// values), which do not change during a solve: a colour pass loads them
// before it waits on its predecessor, so that under programmatic dependent
// launch they arrive while that pass drains.
template <typename T>
struct BellHead {
  static constexpr int kSlots = sizeof(T) == 4 ? 8 : 4;  // as bell_offdiag
  int q0, q1;
  int bc[kSlots];
  T vv[kSlots][9];
};

template <typename T>
__device__ __forceinline__ void bell_head(const BellView<T> &A, int s, int lane, BellHead<T> &h) {
  constexpr int kSlots = BellHead<T>::kSlots;
  h.q0 = __ldg(A.bptr + s);
  h.q1 = __ldg(A.bptr + s + 1);
  const T *va = A.val + 9 * static_cast<size_t>(h.q0) + lane;
#pragma unroll
  for (int u = 0; u < kSlots; ++u) {
    const bool in = h.q0 + 32 * u < h.q1;
    h.bc[u] = in ? __ldg(A.col + h.q0 + 32 * u + lane) : -1;
#pragma unroll
    for (int e = 0; e < 9; ++e) h.vv[u][e] = in ? __ldg(va + (9 * u + e) * 32) : T(0);
  }
}

// bell_offdiag with the first group of slots taken from a loaded head: the
// same slots in the same order, so the same sums bit for bit.
template <typename T, bool kSkip, bool kRel = false>
__device__ __forceinline__ void bell_offdiag_head(const BellView<T> &A, const BellHead<T> &h, int lane,
                                                  const T *__restrict__ x, int skip_from, T acc[3],
                                                  const T *__restrict__ xp = nullptr, int lo = 0, int hi = 0) {
  constexpr int kSlots = BellHead<T>::kSlots;
  acc[0] = acc[1] = acc[2] = T(0);
  {
    bool use[kSlots];
    T xv[kSlots][3];
#pragma unroll
    for (int u = 0; u < kSlots; ++u) {
      use[u] = h.bc[u] >= 0 && (!kSkip || h.bc[u] < skip_from);
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[u][c] = use[u] ? nb_load<kRel>(x, xp, 3 * lo, 3 * hi, 3 * h.bc[u] + c) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u)
      if (use[u])
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[r] = fma(h.vv[u][3 * r + c], xv[u][c], acc[r]);
  }
  for (int q = h.q0 + 32 * kSlots; q < h.q1; q += 32 * kSlots) {
    int bc[kSlots];
    bool in[kSlots], use[kSlots];
    T xv[kSlots][3], vv[kSlots][9];
    const T *va = A.val + 9 * static_cast<size_t>(q) + lane;
#pragma unroll
    for (int u = 0; u < kSlots; ++u) {
      in[u] = q + 32 * u < h.q1;
      bc[u] = in[u] ? __ldg(A.col + q + 32 * u + lane) : -1;
#pragma unroll
      for (int e = 0; e < 9; ++e) vv[u][e] = in[u] ? __ldg(va + (9 * u + e) * 32) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u) {
      use[u] = in[u] && (!kSkip || bc[u] < skip_from);
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[u][c] = use[u] ? nb_load<kRel>(x, xp, 3 * lo, 3 * hi, 3 * bc[u] + c) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u)
      if (use[u])
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[r] = fma(vv[u][3 * r + c], xv[u][c], acc[r]);
  }
}

template <int G, typename T>
__device__ __forceinline__ void reduce3(T acc[3]) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o);
    acc[1] += __shfl_xor_sync(0xffffffffu, acc[1], o);
    acc[2] += __shfl_xor_sync(0xffffffffu, acc[2], o);
  }
}

// The slice's diagonal (or inverted diagonal) blocks, 9 per node, node after
// node, are staged in shared memory: fetched with coalesced loads (lane l
// reads entries l, l + 32, ...) into registers first, so they arrive while
// the off-diagonal sum runs, then stored and read back per node (odd stride
// 9: no bank conflict) instead of 9 strided global loads per lane.
template <typename T>
struct NodeBlocks {
  T v[9];
  int cnt;
};

template <typename T>
__device__ __forceinline__ void fetch_node_blocks(const T *__restrict__ src, int n0, int n1, int lane,
                                                  NodeBlocks<T> &nb) {
  const T *p = src + 9 * static_cast<size_t>(n0);
  nb.cnt = 9 * (n1 - n0);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int e = lane + 32 * k;
    nb.v[k] = e < nb.cnt ? __ldg(p + e) : T(0);
  }
}

template <typename T>
__device__ __forceinline__ void stage_node_blocks(const NodeBlocks<T> &nb, int lane, T *dst /* 288 */) {
  __syncwarp();  // earlier reads of dst by this warp are done
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int e = lane + 32 * k;
    if (e < nb.cnt) dst[e] = nb.v[k];
  }
  __syncwarp();
}

// G lanes per node: a slice holds 32 / G nodes, lane l serves node l / G.
template <typename T, typename BT, int kMode, int G = 1>
__global__ void __launch_bounds__(256, 2) bell_spmv_kernel(BellView<T> A, const T *__restrict__ x,
                                                        T *__restrict__ y,
                                                        const BT *__restrict__ b,
                                                        const int *done) {
  __shared__ T sdiag[8][288];
  if (pass_entry(done)) return;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  T *sd = sdiag[threadIdx.x >> 5];
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslices; s += warps) {
    const int n0 = A.srow[s], n1 = A.srow[s + 1];
    NodeBlocks<T> nb;
    fetch_node_blocks(A.diag, n0, n1, lane, nb);
    T acc[3];
    bell_offdiag<T, false>(A, s, lane, x, 0, acc);
    reduce3<G>(acc);
    stage_node_blocks(nb, lane, sd);
    const int node = n0 + lane / G;
    if ((lane & (G - 1)) == 0 && node < n1) {
      const T *d = sd + 9 * (lane / G);
      const T x0 = x[3 * node], x1 = x[3 * node + 1], x2 = x[3 * node + 2];
      for (int r = 0; r < 3; ++r) {
        T sum = acc[r];
        sum = fma(d[3 * r + 0], x0, sum);
        sum = fma(d[3 * r + 1], x1, sum);
        sum = fma(d[3 * r + 2], x2, sum);
        const int row = 3 * node + r;
        if (kMode == kSpmvSet) y[row] = sum;
        else if (kMode == kSpmvResid) y[row] = T(b[row]) - sum;
        else y[row] += sum;
      }
    }
  }
}

// 3x3 block Gauss-Seidel colour pass: x_I <- (1-w) x_I + w D_I^-1 (b_I - sum_{J != I} A_IJ x_J).
template <typename T, typename BT, bool kZero, int G = 1, bool kRel = false>
__global__ void __launch_bounds__(256, 2) bell_gs_kernel(BellView<T> A, int s_begin, int s_end,
                                                      int node_begin, const BT *__restrict__ b,
                                                      T *__restrict__ x, const T *__restrict__ wts,
                                                      T omega, const int *done,
                                                      const T *__restrict__ nw,
                                                      const T *__restrict__ xprev = nullptr, int node_end = 0) {
  __shared__ T sdinv[8][288];
  const int lane = threadIdx.x & 31;
  const int s = s_begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  // the slice's matrix operands (first group of block slots, inverse
  // diagonal blocks) before the wait on the predecessor: see BellHead
  BellHead<T> h;
  NodeBlocks<T> nb;
  int n0 = 0, n1 = 0;
  if (s < s_end) {
    n0 = __ldg(A.srow + s), n1 = __ldg(A.srow + s + 1);
    bell_head(A, s, lane, h);
    fetch_node_blocks(A.dinv, n0, n1, lane, nb);
  }
  if (pass_entry(done)) return;
  if (s >= s_end) return;
  T *sd = sdinv[threadIdx.x >> 5];
  T acc[3];
  bell_offdiag_head<T, kZero, kRel>(A, h, lane, x, node_begin, acc, xprev, node_begin, node_end);
  reduce3<G>(acc);
  stage_node_blocks(nb, lane, sd);
  const int node = n0 + lane / G;
  if ((lane & (G - 1)) == 0 && node < n1) {
    // a learned scaling per block row (node), else the colour's weight, else omega
    const T w = nw != nullptr ? __ldg(nw + node) : (wts != nullptr ? wts[0] : omega);
    const T r0 = T(b[3 * node]) - acc[0];
    const T r1 = T(b[3 * node + 1]) - acc[1];
    const T r2 = T(b[3 * node + 2]) - acc[2];
    const T *di = sd + 9 * (lane / G);
    for (int r = 0; r < 3; ++r) {
      T nv = di[3 * r] * r0;
      nv = fma(di[3 * r + 1], r1, nv);
      nv = fma(di[3 * r + 2], r2, nv);
      const int row = 3 * node + r;
      x[row] = kZero ? w * nv : (T(1) - w) * x[row] + w * nv;
    }
  }
}

// ---- 3x3 block CSR-vector kernels: G lanes per node row ------------------------
// Coarse block levels (Galerkin elasticity operators) carry 40-70 blocks per
// node row and few nodes per colour. G consecutive lanes share a node row;
// lane j takes blocks rp[I] + j, + j + G, ... (9 values row-major each) and the
// group reduces its three partial sums with shuffles.
template <typename T>
struct BsrvView {
  int nodes;
  const int *__restrict__ rp;    // nodes + 1, in blocks
  const int *__restrict__ bc;    // block column per block
  const T *__restrict__ v;       // 9 per block, row-major
  const T *__restrict__ diag;    // 9 per node
  const T *__restrict__ dinv;    // 9 per node
};

template <typename T, bool kSkip, int G>
__device__ __forceinline__ void bsrv_offdiag(const BsrvView<T> &A, int node, bool valid, int sub,
                                             const T *__restrict__ x, int skip_from, T acc[3]) {
  acc[0] = acc[1] = acc[2] = T(0);
  if (valid) {
    const int k1 = A.rp[node + 1];
    // chunks of 4 blocks per lane: the 4 block-column loads, then the 12
    // gathers, then values and FMAs (two dependent round trips per chunk)
    for (int k0 = A.rp[node] + sub; k0 < k1; k0 += 4 * G) {
      int J[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) J[u] = k0 + u * G < k1 ? __ldg(A.bc + k0 + u * G) : -1;
      T xv[4][3];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool use = J[u] >= 0 && (!kSkip || J[u] < skip_from);
#pragma unroll
        for (int c = 0; c < 3; ++c) xv[u][c] = use ? __ldg(x + 3 * J[u] + c) : T(0);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (J[u] < 0) continue;
        const T *b = A.v + 9 * static_cast<size_t>(k0 + u * G);
#pragma unroll
        for (int r = 0; r < 3; ++r)
          acc[r] = fma(__ldg(b + 3 * r), xv[u][0], fma(__ldg(b + 3 * r + 1), xv[u][1],
                                                        fma(__ldg(b + 3 * r + 2), xv[u][2], acc[r])));
      }
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o, G);
    acc[1] += __shfl_xor_sync(0xffffffffu, acc[1], o, G);
    acc[2] += __shfl_xor_sync(0xffffffffu, acc[2], o, G);
  }
}

// The lane's first chunk of 4 blocks of a node row (block columns and
// values) and, on the row's first lane, its inverse diagonal block: constant
// during a solve, loaded before a colour pass waits on its predecessor.
template <typename T>
struct BsrvHead {
  int k0, k1;
  int J[4];
  T v[4][9];
  T di[9];
};

template <typename T, int G>
__device__ __forceinline__ void bsrv_head(const BsrvView<T> &A, int node, bool valid, int sub, BsrvHead<T> &h) {
  h.k0 = h.k1 = 0;
  if (valid) {
    h.k0 = __ldg(A.rp + node) + sub;
    h.k1 = __ldg(A.rp + node + 1);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int k = h.k0 + u * G;
    const bool in = k < h.k1;
    h.J[u] = in ? __ldg(A.bc + k) : -1;
    const T *bv = A.v + 9 * static_cast<size_t>(in ? k : 0);
#pragma unroll
    for (int e = 0; e < 9; ++e) h.v[u][e] = in ? __ldg(bv + e) : T(0);
  }
  const T *d = A.dinv + 9 * static_cast<size_t>(valid ? node : 0);
#pragma unroll
  for (int e = 0; e < 9; ++e) h.di[e] = valid && sub == 0 ? __ldg(d + e) : T(0);
}

// bsrv_offdiag from a loaded head: the same chunks, the same FMA order.
template <typename T, bool kSkip, int G, bool kRel = false>
__device__ __forceinline__ void bsrv_offdiag_head(const BsrvView<T> &A, const BsrvHead<T> &h,
                                                  const T *__restrict__ x, int skip_from, T acc[3],
                                                  const T *__restrict__ xp = nullptr, int lo = 0, int hi = 0) {
  acc[0] = acc[1] = acc[2] = T(0);
  {
    T xv[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool use = h.J[u] >= 0 && (!kSkip || h.J[u] < skip_from);
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[u][c] = use ? nb_load<kRel>(x, xp, 3 * lo, 3 * hi, 3 * h.J[u] + c) : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (h.J[u] < 0) continue;
#pragma unroll
      for (int r = 0; r < 3; ++r)
        acc[r] = fma(h.v[u][3 * r], xv[u][0], fma(h.v[u][3 * r + 1], xv[u][1], fma(h.v[u][3 * r + 2], xv[u][2], acc[r])));
    }
  }
  for (int k0 = h.k0 + 4 * G; k0 < h.k1; k0 += 4 * G) {
    int J[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) J[u] = k0 + u * G < h.k1 ? __ldg(A.bc + k0 + u * G) : -1;
    T xv[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool use = J[u] >= 0 && (!kSkip || J[u] < skip_from);
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[u][c] = use ? nb_load<kRel>(x, xp, 3 * lo, 3 * hi, 3 * J[u] + c) : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (J[u] < 0) continue;
      const T *b = A.v + 9 * static_cast<size_t>(k0 + u * G);
#pragma unroll
      for (int r = 0; r < 3; ++r)
        acc[r] = fma(__ldg(b + 3 * r), xv[u][0], fma(__ldg(b + 3 * r + 1), xv[u][1],
                                                      fma(__ldg(b + 3 * r + 2), xv[u][2], acc[r])));
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o, G);
    acc[1] += __shfl_xor_sync(0xffffffffu, acc[1], o, G);
    acc[2] += __shfl_xor_sync(0xffffffffu, acc[2], o, G);
  }
}

template <typename T, typename BT, bool kZero, int G, bool kRel = false>
__global__ void __launch_bounds__(256) bsrv_gs_kernel(BsrvView<T> A, int node_begin, int node_end,
                                                      const BT *__restrict__ b, T *__restrict__ x,
                                                      const T *__restrict__ wts, T omega,
                                                      const int *done, const T *__restrict__ nw,
                                                      const T *__restrict__ xprev = nullptr) {
  const int sub = threadIdx.x & (G - 1);
  const int node = node_begin + (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = node < node_end;
  // matrix operands first (constant during a solve), then the wait on the
  // predecessor pass, then the iterate
  BsrvHead<T> h;
  bsrv_head<T, G>(A, node, valid, sub, h);
  if (pass_entry(done)) return;
  T acc[3];
  bsrv_offdiag_head<T, kZero, G, kRel>(A, h, x, node_begin, acc, xprev, node_begin, node_end);
  if (valid && sub == 0) {
    const T w = nw != nullptr ? __ldg(nw + node) : (wts != nullptr ? wts[0] : omega);
    const T r0 = T(b[3 * node]) - acc[0];
    const T r1 = T(b[3 * node + 1]) - acc[1];
    const T r2 = T(b[3 * node + 2]) - acc[2];
    const T *di = h.di;
    for (int r = 0; r < 3; ++r) {
      T nv = di[3 * r] * r0;
      nv = fma(di[3 * r + 1], r1, nv);
      nv = fma(di[3 * r + 2], r2, nv);
      const int row = 3 * node + r;
      x[row] = kZero ? w * nv : (T(1) - w) * x[row] + w * nv;
    }
  }
}

template <typename T, typename BT, int kMode, int G>
__global__ void __launch_bounds__(256) bsrv_spmv_kernel(BsrvView<T> A, const T *__restrict__ x,
                                                        T *__restrict__ y,
                                                        const BT *__restrict__ b,
                                                        const int *done) {
  if (pass_entry(done)) return;
  const int sub = threadIdx.x & (G - 1);
  const int groups = (gridDim.x * blockDim.x) / G;
  const int first = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int trips = (A.nodes + groups - 1) / groups;
  for (int t = 0; t < trips; ++t) {
    const int node = first + t * groups;
    const bool valid = node < A.nodes;
    T acc[3];
    bsrv_offdiag<T, false, G>(A, node, valid, sub, x, 0, acc);
    if (valid && sub == 0) {
      const T *d = A.diag + 9 * static_cast<size_t>(node);
      const T x0 = x[3 * node], x1 = x[3 * node + 1], x2 = x[3 * node + 2];
      for (int r = 0; r < 3; ++r) {
        T sum = acc[r];
        sum = fma(d[3 * r + 0], x0, sum);
        sum = fma(d[3 * r + 1], x1, sum);
        sum = fma(d[3 * r + 2], x2, sum);
        const int row = 3 * node + r;
        if (kMode == kSpmvSet) y[row] = sum;
        else if (kMode == kSpmvResid) y[row] = T(b[row]) - sum;
        else y[row] += sum;
      }
    }
  }
}

// ---- reductions -------------------------------------------------------------
template <int kN>
__device__ __forceinline__ void block_sum(double (&v)[kN], double *smem /* 32*kN */) {
#pragma unroll
  for (int i = 0; i < kN; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < kN; ++i) smem[warp * kN + i] = v[i];
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < kN; ++i) {
      v[i] = lane < nw ? smem[lane * kN + i] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
    }
  }
}

// Deterministic grid reduction: each block writes its partial sums, the last
// block to arrive adds all partials in a fixed order. Returns true in every
// thread of the last block, with v[] holding the totals in thread 0.
template <int kN>
__device__ __forceinline__ bool grid_sum(double (&v)[kN], double *partials, unsigned int *ticket,
                                         double *smem) {
  block_sum<kN>(v, smem);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < kN; ++i) partials[blockIdx.x * kN + i] = v[i];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double t[kN];
#pragma unroll
  for (int i = 0; i < kN; ++i) t[i] = 0.0;
  for (unsigned int bk = threadIdx.x; bk < gridDim.x; bk += blockDim.x)
#pragma unroll
    for (int i = 0; i < kN; ++i)
      t[i] += reinterpret_cast<volatile double *>(partials)[bk * kN + i];
  block_sum<kN>(t, smem);
#pragma unroll
  for (int i = 0; i < kN; ++i) v[i] = t[i];
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// ---- CG kernels (FP64 outer iteration) --------------------------------------
__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// Ap = A p and pAp = p . Ap; the last block sets alpha = rho / pAp.
static __global__ void __launch_bounds__(256) cg_spmv_pap_kernel(SellView<double> A,
                                                          const double *__restrict__ p,
                                                          double *__restrict__ ap, CgState *st,
                                                          double *partials) {
  __shared__ double smem[32];
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslices; s += warps) {
    double sum = sell_offdiag<double, false>(A, s, lane, p, 0);
    const int row = A.srow[s] + lane;
    if (row < A.srow[s + 1]) {
      const double pr = p[row];
      sum = fma(A.diag[row], pr, sum);
      ap[row] = sum;
      acc[0] = fma(pr, sum, acc[0]);
    }
  }
  if (grid_sum<1>(acc, partials, &st->ticket, smem) && threadIdx.x == 0) {
    const double pap = acc[0];
    st->pAp = pap;
    if (!finite_d(pap) || pap == 0.0) {
      st->status = pap == 0.0 ? kCgBreakdown : kCgNotFinite;
      st->done = 1;
      st->iterations = st->iter;
    }
    st->alpha = st->rho / pap;
  }
}

// Same as cg_spmv_pap_kernel for a 3x3-blocked operator in BELL-32 with G
// lanes per node (a slice holds 32 / G nodes; the lanes of a node add their
// partial sums with shuffles).
template <int G>
__global__ void __launch_bounds__(256, 2) cg_bell_spmv_pap_kernel(BellView<double> A,
                                                               const double *__restrict__ p,
                                                               double *__restrict__ ap, CgState *st,
                                                               double *partials) {
  __shared__ double smem[32];
  __shared__ double sdiag[8][288];
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  double *sd = sdiag[threadIdx.x >> 5];
  double acc[1] = {0.0};
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslices; s += warps) {
    const int n0 = A.srow[s], n1 = A.srow[s + 1];
    NodeBlocks<double> nb;
    fetch_node_blocks(A.diag, n0, n1, lane, nb);
    double o[3];
    bell_offdiag<double, false>(A, s, lane, p, 0, o);
    reduce3<G>(o);
    stage_node_blocks(nb, lane, sd);
    const int node = n0 + lane / G;
    if ((lane & (G - 1)) == 0 && node < n1) {
      const double *d = sd + 9 * (lane / G);
      const double x0 = p[3 * node], x1 = p[3 * node + 1], x2 = p[3 * node + 2];
      for (int r = 0; r < 3; ++r) {
        double sum = o[r];
        sum = fma(d[3 * r + 0], x0, sum);
        sum = fma(d[3 * r + 1], x1, sum);
        sum = fma(d[3 * r + 2], x2, sum);
        ap[3 * node + r] = sum;
        acc[0] = fma(p[3 * node + r], sum, acc[0]);
      }
    }
  }
  if (grid_sum<1>(acc, partials, &st->ticket, smem) && threadIdx.x == 0) {
    const double pap = acc[0];
    st->pAp = pap;
    if (!finite_d(pap) || pap == 0.0) {
      st->status = pap == 0.0 ? kCgBreakdown : kCgNotFinite;
      st->done = 1;
      st->iterations = st->iter;
    }
    st->alpha = st->rho / pap;
  }
}

// x += alpha p; r -= alpha Ap; rr = r . r; convergence test on rr / bb.
static __global__ void __launch_bounds__(256) cg_update_xr_kernel(int n, double *__restrict__ x,
                                                           double *__restrict__ r,
                                                           const double *__restrict__ p,
                                                           const double *__restrict__ ap,
                                                           CgState *st, double *partials) {
  __shared__ double smem[32];
  if (st->done) return;
  const double alpha = st->alpha;
  double acc[1] = {0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, ap[i], r[i]);
    r[i] = ri;
    acc[0] = fma(ri, ri, acc[0]);
  }
  if (grid_sum<1>(acc, partials, &st->ticket, smem) && threadIdx.x == 0) {
    st->rr = acc[0];
    const double ratio = acc[0] / st->bb;
    st->ratio = ratio;
    if (!finite_d(ratio)) {
      st->status = kCgNotFinite;
      st->done = 1;
      st->iterations = st->iter;
    } else if (ratio < st->tol2) {
      st->status = kCgConverged;
      st->done = 1;
      st->iterations = st->iter;  // 0-based, as the reference counts
    } else if (st->iter + 1 >= st->max_iter) {
      st->status = kCgMaxIter;
      st->done = 1;
      st->iterations = st->max_iter;
    }
    st->iter += 1;
  }
}

// rho_new = r . z (and r . z_old for the flexible variant); the last block
// sets beta = (rho_new - r.z_old) / rho (Polak-Ribiere) or rho_new / rho.
template <typename ZT>
__global__ void __launch_bounds__(256) cg_dot_rz_kernel(int n, const double *__restrict__ r,
                                                        const ZT *__restrict__ z,
                                                        const ZT *__restrict__ z_old, CgState *st,
                                                        double *partials) {
  __shared__ double smem[64];
  if (st->done) return;
  double acc[2] = {0.0, 0.0};
  const int stride = gridDim.x * blockDim.x;
  const bool flex = z_old != nullptr;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double ri = r[i];
    acc[0] = fma(ri, double(z[i]), acc[0]);
    if (flex) acc[1] = fma(ri, double(z_old[i]), acc[1]);
  }
  if (grid_sum<2>(acc, partials, &st->ticket, smem) && threadIdx.x == 0) {
    st->rho_new = acc[0];
    st->rz_old = acc[1];
    st->beta = (flex ? (acc[0] - acc[1]) : acc[0]) / st->rho;
    st->rho = acc[0];
  }
}

// p = z + beta p.
template <typename ZT>
__global__ void __launch_bounds__(256) cg_update_p_kernel(int n, const ZT *__restrict__ z,
                                                          double *__restrict__ p,
                                                          const CgState *st) {
  if (st->done) return;
  const double beta = st->beta;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    p[i] = fma(beta, p[i], double(z[i]));
}

// Start of the solve: p = z; bb = b.b, rho = r.z, rr = r.r.
template <typename ZT>
__global__ void __launch_bounds__(256) cg_init_kernel(int n, const double *__restrict__ b,
                                                      const double *__restrict__ r,
                                                      const ZT *__restrict__ z,
                                                      double *__restrict__ p, CgState *st,
                                                      double *partials) {
  __shared__ double smem[96];
  double acc[3] = {0.0, 0.0, 0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double zi = double(z[i]), ri = r[i], bi = b[i];
    p[i] = zi;
    acc[0] = fma(bi, bi, acc[0]);
    acc[1] = fma(ri, zi, acc[1]);
    acc[2] = fma(ri, ri, acc[2]);
  }
  if (grid_sum<3>(acc, partials, &st->ticket, smem) && threadIdx.x == 0) {
    st->bb = acc[0];
    st->rho = acc[1];
    st->rr = acc[2];
    st->ratio = acc[2] / acc[0];
    st->iter = 0;
    st->done = 0;
    st->status = kCgRunning;
    st->iterations = 0;
    if (!finite_d(st->ratio)) {
      st->status = kCgNotFinite;
      st->done = 1;
    } else if (st->ratio < st->tol2) {
      st->status = kCgInitialConverged;
      st->done = 1;
    }
  }
}

// bb = b.b only (zero right-hand side test).
static __global__ void __launch_bounds__(256) dot_self_kernel(int n, const double *__restrict__ b,
                                                       double *out, double *partials,
                                                       unsigned int *ticket) {
  __shared__ double smem[32];
  double acc[1] = {0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    acc[0] = fma(b[i], b[i], acc[0]);
  if (grid_sum<1>(acc, partials, ticket, smem) && threadIdx.x == 0) *out = acc[0];
}

// ---- coarsest level: x = A^-1 b with the inverse formed at setup in FP64
//      and stored in the V-cycle's precision, one warp per row, FP64 sums.
template <typename BT, typename VT>
__global__ void __launch_bounds__(256) dense_solve_kernel(int n, const VT *__restrict__ ainv,
                                                          const BT *__restrict__ b,
                                                          VT *__restrict__ x, const int *done) {
  if (pass_entry(done)) return;
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const VT *a = ainv + static_cast<size_t>(row) * n;
  double sum = 0.0;
  for (int j = lane; j < n; j += 32) sum = fma(double(__ldg(a + j)), double(b[j]), sum);
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
  if (lane == 0) x[row] = VT(sum);
}

// ---- coarsest level, packed symmetric inverse (large dense levels) -----------
// Only the lower triangle of A^-1 is stored, as kDenseTile x kDenseTile tiles
// (zero beyond n), tile (I, J), I >= J, at (I (I + 1) / 2 + J) * kDenseTile^2.
// One 256-thread CTA per tile reads it once and produces both of its
// contributions: A_IJ x_J for the rows of tile row I and, off the diagonal,
// A_IJ^T x_I for the rows of tile row J. Each lands in its own slot
// partial[I][J] (resp. partial[J][I]) of kDenseTile FP64 values; the reduce
// kernel sums a row's T slots in slot order, so x = A^-1 b comes out the same
// on every run while the inverse crosses HBM once, at half the bytes of the
// full matrix.
// Inside a tile, thread t owns the 4 x 4 block of rows 4 (t / 16) .. +3 and
// columns 4 (t % 16) .. +3, in registers: its 16 values are stored as 16-byte
// chunks, chunk k of every thread of the CTA contiguous (k * 256 + t), so each
// load instruction of a warp reads 512 contiguous bytes. Row sums reduce over
// the 16 lanes that share a row block (shuffles), column sums over the 16 row
// blocks through shared memory in a fixed order.
constexpr int kDenseTile = 64;

// Offset of element (r, c) of a tile in the packed layout above.
template <typename VT>
__host__ __device__ __forceinline__ int dense_tile_offset(int r, int c) {
  constexpr int kV = 16 / sizeof(VT);
  const int t = (r / 4) * 16 + c / 4, e = (r % 4) * 4 + c % 4;
  return ((e / kV) * 256 + t) * kV + e % kV;
}

// Offset (in halves) of element (r, c) of an FP16 tile, the layout the
// tensor-core apply reads with ldmatrix: 4 x 4 blocks of 16 x 16, block
// (ib, kb) at (4 ib + kb) * 256, each four row-major 8 x 8 matrices (rh, ch)
// at (2 rh + ch) * 64.
__host__ __device__ __forceinline__ int dense_mma_offset(int r, int c) {
  const int b = (r >> 4) * 4 + (c >> 4);
  const int m = ((r >> 3) & 1) * 2 + ((c >> 3) & 1);
  return b * 256 + m * 64 + (r & 7) * 8 + (c & 7);
}

__device__ __forceinline__ void dense_tile_of(long long t, int &I, int &J) {
  I = static_cast<int>((sqrt(8.0 * static_cast<double>(t) + 1.0) - 1.0) * 0.5);
  while (static_cast<long long>(I) * (I + 1) / 2 > t) --I;
  while (static_cast<long long>(I + 1) * (I + 2) / 2 <= t) ++I;
  J = static_cast<int>(t - static_cast<long long>(I) * (I + 1) / 2);
}

// Each CTA takes dense_tiles_per_cta<ST>() consecutive tiles and issues the
// loads of all of them before computing any, to keep more bytes in flight per
// SM: 2 tiles of FP32 or FP64 (64 KB / 128 KB).
template <typename ST>
__host__ __device__ constexpr int dense_tiles_per_cta() {
  return 2;
}
constexpr int kDenseTilesPerCta = 2;

// ST: the storage type of the tiles, the V-cycle's precision (FP32 or FP64;
// FP16 tiles have their own layout and the tensor-core apply,
// dense_mma_kernel). `scales`, when given, multiplies each tile's 4-term
// products once.
template <typename BT, typename VT, typename ST = VT>
__global__ void __launch_bounds__(256) dense_tile_kernel(int n, int tiles, const ST *__restrict__ packed,
                                                         const BT *__restrict__ b, double *__restrict__ partial,
                                                         const int *done, const float *__restrict__ scales = nullptr) {
  static_assert(sizeof(ST) >= 4, "FP16 tiles are applied by dense_mma_kernel");
  if (pass_entry(done)) return;
  constexpr int TB = kDenseTile, kV = 16 / sizeof(ST), kChunks = 16 / kV, kT = dense_tiles_per_cta<ST>();
  __shared__ double colpart[16][TB];
  const long long total = static_cast<long long>(tiles) * (tiles + 1) / 2;
  const long long t0 = static_cast<long long>(blockIdx.x) * kT;
  const int tid = threadIdx.x, rb = tid >> 4, cb = tid & 15;
  union Chunk {
    uint4 u;
    ST v[kV];
  };
  Chunk w[kT][kChunks];
#pragma unroll
  for (int tt = 0; tt < kT; ++tt) {
    if (t0 + tt >= total) break;
    const uint4 *tile = reinterpret_cast<const uint4 *>(packed + (t0 + tt) * TB * TB);
#pragma unroll
    for (int k = 0; k < kChunks; ++k) w[tt][k].u = __ldg(tile + k * 256 + tid);
  }
#pragma unroll
  for (int tt = 0; tt < kT; ++tt) {
    if (t0 + tt >= total) break;  // uniform over the CTA
    int I, J;
    dense_tile_of(t0 + tt, I, J);
    const double sc = scales != nullptr ? double(__ldg(scales + t0 + tt)) : 1.0;
    // a thread's 4-term products in the V-cycle's precision, everything
    // across threads in FP64
    VT xr[4], xc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = I * TB + rb * 4 + i, c = J * TB + cb * 4 + i;
      xr[i] = r < n ? VT(b[r]) : VT(0);
      xc[i] = c < n ? VT(b[c]) : VT(0);
    }
    VT rv[4] = {VT(0), VT(0), VT(0), VT(0)}, cv[4] = {VT(0), VT(0), VT(0), VT(0)};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const VT a = VT(w[tt][(i * 4 + j) / kV].v[(i * 4 + j) % kV]);
        rv[i] = fma(a, xc[j], rv[i]);
        cv[j] = fma(a, xr[i], cv[j]);
      }
    double rs[4], cs[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      rs[i] = double(rv[i]) * sc;
      cs[i] = double(cv[i]) * sc;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) rs[i] += __shfl_xor_sync(0xffffffffu, rs[i], o);
    }
    if (cb == 0)
#pragma unroll
      for (int i = 0; i < 4; ++i) partial[(static_cast<size_t>(I) * tiles + J) * TB + rb * 4 + i] = rs[i];
    if (I != J) {  // uniform over the CTA
      __syncthreads();  // colpart of the previous tile has been read
#pragma unroll
      for (int j = 0; j < 4; ++j) colpart[rb][cb * 4 + j] = cs[j];
      __syncthreads();
      if (tid < TB) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q) sum += colpart[q][tid];
        partial[(static_cast<size_t>(J) * tiles + I) * TB + tid] = sum;
      }
    }
  }
}

// One block per tile row: thread (g, r) sums slots K = g, g + 4, ... of row
// r in order, then the four groups are added in group order.
template <typename VT, typename PT = double>
__global__ void __launch_bounds__(256) dense_reduce_kernel(int n, int tiles, const PT *__restrict__ partial,
                                                           VT *__restrict__ x, const int *done) {
  if (pass_entry(done)) return;
  __shared__ double part[4][kDenseTile];
  const int I = blockIdx.x, r = threadIdx.x % kDenseTile, g = threadIdx.x / kDenseTile;
  const PT *p = partial + static_cast<size_t>(I) * tiles * kDenseTile + r;
  double sum = 0.0;
#pragma unroll 8
  for (int K = g; K < tiles; K += 4) sum += double(__ldg(p + static_cast<size_t>(K) * kDenseTile));
  part[g][r] = sum;
  __syncthreads();
  const int i = I * kDenseTile + threadIdx.x;
  if (threadIdx.x < kDenseTile && i < n)
    x[i] = VT(((part[0][threadIdx.x] + part[1][threadIdx.x]) + part[2][threadIdx.x]) + part[3][threadIdx.x]);
}

template <typename ST>
__device__ __forceinline__ ST to_storage(double v) {
  return ST(v);
}
template <>
__device__ __forceinline__ __half to_storage<__half>(double v) {
  return __float2half_rn(static_cast<float>(v));
}

// Packs the row-major FP64 inverse (n x n) into lower-triangle tiles of ST.
// With `scales` (ST = __half) every tile is stored divided by its largest
// magnitude over 16384 (that factor goes to scales[tile]), so the values use
// FP16's normal range with 11 significant bits.
template <typename ST>
__global__ void dense_pack_kernel(int n, const double *__restrict__ full, ST *__restrict__ packed,
                                  float *__restrict__ scales = nullptr) {
  constexpr int TB = kDenseTile;
  __shared__ double red[32];
  int I, J;
  dense_tile_of(blockIdx.x, I, J);
  ST *tile = packed + static_cast<long long>(blockIdx.x) * TB * TB;
  double inv_scale = 1.0;
  if (scales != nullptr) {
    double m = 0.0;
    for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
      const int r = I * TB + e / TB, c = J * TB + e % TB;
      if (r < n && c < n) m = fmax(m, fabs(full[static_cast<size_t>(r) * n + c]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = 0.0;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) mm = fmax(mm, red[w]);
      red[0] = mm > 0.0 ? mm / 16384.0 : 1.0;
      scales[blockIdx.x] = static_cast<float>(red[0]);
    }
    __syncthreads();
    inv_scale = 1.0 / double(scales[blockIdx.x]);
  }
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int lr = e / TB, lc = e % TB, r = I * TB + lr, c = J * TB + lc;
    const double v = (r < n && c < n) ? full[static_cast<size_t>(r) * n + c] * inv_scale : 0.0;
    // FP16 tiles are read by the tensor-core apply (dense_mma_kernel)
    const int off = sizeof(ST) == 2 ? dense_mma_offset(lr, lc) : dense_tile_offset<ST>(lr, lc);
    tile[off] = to_storage<ST>(v);
  }
}

// ---- Jacobi smoothers (DampedJacobiSmoother / BlockJacobiSmoother) ----------
// x <- x + w D^-1 v with v = b - A x (the residual of the current x), or,
// from an implicit zero x, x <- w D^-1 b. D^-1: 1 / a_ii per row, or the 3x3
// inverse diagonal block per node (row-major, 9 per node).
template <typename T, typename BT, bool kZero>
__global__ void __launch_bounds__(256) jacobi_kernel(int n, const T *__restrict__ dinv,
                                                     const BT *__restrict__ v, T *__restrict__ x, T w,
                                                     const int *done) {
  if (pass_entry(done)) return;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const T c = T(v[i]) * dinv[i];
    x[i] = kZero ? w * c : x[i] + w * c;
  }
}

template <typename T, typename BT, bool kZero>
__global__ void __launch_bounds__(256) block_jacobi_kernel(int nodes, const T *__restrict__ dinv,
                                                           const BT *__restrict__ v, T *__restrict__ x,
                                                           T w, const int *done) {
  if (pass_entry(done)) return;
  const int stride = gridDim.x * blockDim.x;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nodes; I += stride) {
    const T r0 = T(v[3 * I]), r1 = T(v[3 * I + 1]), r2 = T(v[3 * I + 2]);
    const T *d = dinv + 9 * static_cast<size_t>(I);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      T sum = d[3 * r] * r0;
      sum = fma(d[3 * r + 1], r1, sum);
      sum = fma(d[3 * r + 2], r2, sum);
      const int row = 3 * I + r;
      x[row] = kZero ? w * sum : x[row] + w * sum;
    }
  }
}

// IdentityPreconditioner::apply: x = v (with a precision conversion).
template <typename T, typename BT>
__global__ void convert_kernel(int n, const BT *__restrict__ v, T *__restrict__ x, const int *done) {
  if (pass_entry(done)) return;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = T(v[i]);
}

// ---- permutation between the caller's order and the internal colour order.
template <typename T, typename U>
__global__ void gather_kernel(int n, const int *__restrict__ src_of, const T *__restrict__ in,
                              U *__restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = U(in[src_of[i]]);
}
template <typename T, typename U>
__global__ void scatter_kernel(int n, const int *__restrict__ dst_of, const T *__restrict__ in,
                               U *__restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[dst_of[i]] = U(in[i]);
}

// out = a - z (the error after one preconditioner step, e1 = e0 - M A e0)
template <typename ZT>
__global__ void sub_kernel(int n, const double *__restrict__ a, const ZT *__restrict__ z,
                           double *__restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = a[i] - double(z[i]);
}

template <typename T>
__global__ void fill_kernel(int n, T *__restrict__ x, T v) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = v;
}

}  // namespace gsb
