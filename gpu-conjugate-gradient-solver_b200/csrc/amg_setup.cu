// Smoothed-aggregation setup on the GPU.
//
// One coarsening step per level, every part on the device:
//   node couplings (Frobenius norms of the block entries)  -> strength test
//   -> distance-2 maximal independent set by max propagation (rounds)
//   -> aggregates (roots, their strong neighbours, strongest-neighbour join,
//      singletons) -> tentative prolongator (normalised piecewise constants)
//   -> filtered diagonal and Gershgorin bound -> smoothed prolongator
//   -> R = P^T -> Ac = R (A P).
// The arithmetic and the order of every floating-point sum are those of
// sa_coarsen (setup.cc) with aggregation 1, and this file is compiled without
// FMA contraction, so the host build of the same hierarchy is its bit-exact
// check. Layout: plain CSR (int32 row pointers and columns, FP64 values),
// rows sorted by column. Per-node and per-row steps run one thread per item;
// the two sparse products run one warp per output row with an open-addressing
// hash table per warp in shared memory, adding the products of a row in the
// host's order (A's entries in order, each B row in order).
#include "amg_setup.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "solver.h"

#define SCK(x) ::gsb::cuda_check((x), #x)

namespace gsb {
namespace {

// ---------------------------------------------------------------------------
// stream-ordered device buffers
// ---------------------------------------------------------------------------
template <typename T>
class DBuf {
 public:
  DBuf() = default;
  DBuf(size_t n, cudaStream_t s) { alloc(n, s); }
  ~DBuf() { release(); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr, o.n_ = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_, n_ = o.n_, s_ = o.s_;
      o.p_ = nullptr, o.n_ = 0;
    }
    return *this;
  }
  void alloc(size_t n, cudaStream_t s) {
    release();
    s_ = s;
    n_ = n;
    SCK(cudaMallocAsync(reinterpret_cast<void **>(&p_), std::max<size_t>(n, 1) * sizeof(T), s));
  }
  void release() {
    if (p_ != nullptr) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
  }
  T *get() const { return p_; }
  size_t size() const { return n_; }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

struct DCsr {
  int rows = 0, cols = 0, nnz = 0;
  DBuf<int> rp, ci;
  DBuf<double> v;
};

inline int grid_for(long long items, int per_block = 256) {
  long long b = (items + per_block - 1) / per_block;
  return static_cast<int>(std::max<long long>(1, std::min<long long>(b, 1LL << 30)));
}

void check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("GPU setup: ") + what + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// exclusive scan of n ints into out[0..n]; out[n] is the total
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const int *__restrict__ in, int *__restrict__ out,
                                                                 int n, int *__restrict__ tile_sums) {
  __shared__ int warp_sums[kScanThreads / 32];
  const long long base = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
  int x[kScanItems];
  int sum = 0;
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    const long long i = base + t;
    x[t] = i < n ? in[i] : 0;  // element n (and beyond) counts 0
    sum += x[t];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  int run = incl - sum + (warp > 0 ? warp_sums[warp - 1] : 0);
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    const long long i = base + t;
    if (i <= n) out[i] = run;
    run += x[t];
  }
  if (threadIdx.x == kScanThreads - 1) tile_sums[blockIdx.x] = warp_sums[kScanThreads / 32 - 1];
}

__global__ void scan_add_kernel(int *__restrict__ out, int n, const int *__restrict__ tile_offsets) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i <= n) out[i] += tile_offsets[i / kScanTile];
}

void scan_into(const int *in, int *out, int n, cudaStream_t s) {
  const int tiles = static_cast<int>((static_cast<long long>(n) + kScanTile) / kScanTile);  // covers 0..n
  DBuf<int> sums(tiles, s);
  scan_tile_kernel<<<tiles, kScanThreads, 0, s>>>(in, out, n, sums.get());
  check_launch("scan");
  if (tiles > 1) {
    DBuf<int> offs(static_cast<size_t>(tiles) + 1, s);
    scan_into(sums.get(), offs.get(), tiles, s);
    scan_add_kernel<<<grid_for(static_cast<long long>(n) + 1), 256, 0, s>>>(out, n, offs.get());
    check_launch("scan add");
  }
}

// Returns the total (a host-synchronising read of out[n]).
int scan_total(const int *in, int *out, int n, cudaStream_t s) {
  scan_into(in, out, n, s);
  int total = 0;
  SCK(cudaMemcpyAsync(&total, out + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  if (total < 0) throw std::runtime_error("GPU setup: more than 2^31 entries");
  return total;
}

// ---------------------------------------------------------------------------
// node couplings and strength
// ---------------------------------------------------------------------------
constexpr int kMaxBlock = 8;

// Merges the `block` sorted rows of node i by node column. Per node column
// the squares are summed row after row, each row in stored order (the host's
// order). Counting pass when nci == nullptr.
__global__ void couplings_kernel(int nn, int block, const int *__restrict__ rp, const int *__restrict__ ci,
                                 const double *__restrict__ v, int *__restrict__ cnt, const int *__restrict__ nrp,
                                 int *__restrict__ nci, double *__restrict__ nw, double *__restrict__ nd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  int ptr[kMaxBlock], end[kMaxBlock];
  for (int r = 0; r < block; ++r) {
    ptr[r] = rp[block * i + r];
    end[r] = rp[block * i + r + 1];
  }
  const int out = nci != nullptr ? nrp[i] : 0;
  int count = 0;
  double dsum = 0.0;
  for (;;) {
    int j = INT_MAX;
    for (int r = 0; r < block; ++r)
      if (ptr[r] < end[r]) j = min(j, ci[ptr[r]] / block);
    if (j == INT_MAX) break;
    double acc = 0.0;
    for (int r = 0; r < block; ++r)
      while (ptr[r] < end[r] && ci[ptr[r]] / block == j) {
        const double x = v[ptr[r]];
        acc += x * x;
        ++ptr[r];
      }
    if (j == i) {
      dsum = acc;
    } else {
      if (nci != nullptr) {
        nci[out + count] = j;
        nw[out + count] = sqrt(acc);
      }
      ++count;
    }
  }
  if (nci != nullptr) nd[i] = sqrt(dsum);
  else cnt[i] = count;
}

__global__ void strength_kernel(int nn, const int *__restrict__ nrp, const int *__restrict__ nci,
                                const double *__restrict__ nw, const double *__restrict__ nd, double eps2,
                                unsigned char *__restrict__ strong, int *__restrict__ nstrong) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  int c = 0;
  for (int k = nrp[i]; k < nrp[i + 1]; ++k) {
    const bool s = nw[k] * nw[k] >= eps2 * nd[i] * nd[nci[k]];
    strong[k] = s ? 1 : 0;
    c += s ? 1 : 0;
  }
  nstrong[i] = c;
}

// ---------------------------------------------------------------------------
// distance-2 maximal independent set
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t priority_of(uint32_t v) {
  v ^= v >> 16;
  v *= 0x85ebca6bu;
  v ^= v >> 13;
  v *= 0xc2b2ae35u;
  v ^= v >> 16;
  return v;
}

__device__ __forceinline__ uint64_t mis_key(const unsigned char *state, int i) {
  return (static_cast<uint64_t>(state[i]) << 32) | priority_of(static_cast<uint32_t>(i));
}

__device__ __forceinline__ void count_flag(bool flag, int *counter) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if ((threadIdx.x & 31) == 0 && m != 0) atomicAdd(counter, __popc(m));
}

__global__ void mis_init_kernel(int nn, const int *__restrict__ nstrong, unsigned char *__restrict__ state,
                                int *__restrict__ undecided) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < nn && nstrong[i] != 0;
  if (i < nn) state[i] = live ? 1 : 0;
  count_flag(live, undecided);
}

// First pass (t_in == nullptr): largest key over the closed strong
// neighbourhood; second pass: the same over the first pass's results.
__global__ void mis_max_kernel(int nn, const int *__restrict__ nrp, const int *__restrict__ nci,
                               const unsigned char *__restrict__ strong, const unsigned char *__restrict__ state,
                               const uint64_t *__restrict__ t_in, uint64_t *__restrict__ t_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  uint64_t m = t_in != nullptr ? t_in[i] : mis_key(state, i);
  for (int k = nrp[i]; k < nrp[i + 1]; ++k) {
    if (!strong[k]) continue;
    const uint64_t u = t_in != nullptr ? t_in[nci[k]] : mis_key(state, nci[k]);
    m = u > m ? u : m;
  }
  t_out[i] = m;
}

__global__ void mis_decide_kernel(int nn, unsigned char *__restrict__ state, const uint64_t *__restrict__ t2,
                                  int *__restrict__ undecided) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool still = false;
  if (i < nn && state[i] == 1) {
    const uint64_t own = (1ull << 32) | priority_of(static_cast<uint32_t>(i));
    if (t2[i] == own) state[i] = 2;
    else if ((t2[i] >> 32) == 2) state[i] = 0;
    else still = true;
  }
  count_flag(still, undecided);
}

// ---------------------------------------------------------------------------
// aggregates
// ---------------------------------------------------------------------------
__global__ void state_flag_kernel(int nn, const unsigned char *__restrict__ state, unsigned char want,
                                  int *__restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) flag[i] = state[i] == want ? 1 : 0;
}

__global__ void agg_init_kernel(int nn, const int *__restrict__ nstrong, const unsigned char *__restrict__ state,
                                const int *__restrict__ rid, int *__restrict__ agg, int *__restrict__ claim) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  agg[i] = nstrong[i] == 0 ? -2 : (state[i] == 2 ? rid[i] : -1);
  claim[i] = INT_MAX;
}

// Each non-root strong neighbour of a root goes to the lowest-numbered root
// that claims it (roots are numbered in index order).
__global__ void claim_kernel(int nn, const int *__restrict__ nrp, const int *__restrict__ nci,
                             const unsigned char *__restrict__ strong, const unsigned char *__restrict__ state,
                             const int *__restrict__ agg, int *__restrict__ claim) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn || state[i] != 2) return;
  for (int k = nrp[i]; k < nrp[i + 1]; ++k)
    if (strong[k] && agg[nci[k]] == -1) atomicMin(claim + nci[k], agg[i]);
}

__global__ void claim_apply_kernel(int nn, int *__restrict__ agg, const int *__restrict__ claim) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn && agg[i] == -1 && claim[i] != INT_MAX) agg[i] = claim[i];
}

// A node still free joins the aggregate of its strongest strongly coupled
// aggregated neighbour (the first in column order on ties).
__global__ void join_kernel(int nn, const int *__restrict__ nrp, const int *__restrict__ nci,
                            const double *__restrict__ nw, const unsigned char *__restrict__ strong,
                            const int *__restrict__ agg1, int *__restrict__ agg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn || agg1[i] != -1) return;
  int best = -1;
  double bw = -1.0;
  for (int k = nrp[i]; k < nrp[i + 1]; ++k)
    if (strong[k] && agg1[nci[k]] >= 0 && nw[k] > bw) bw = nw[k], best = agg1[nci[k]];
  if (best >= 0) agg[i] = best;
}

__global__ void free_flag_kernel(int nn, const int *__restrict__ agg, int *__restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) flag[i] = agg[i] == -1 ? 1 : 0;
}

__global__ void singleton_kernel(int nn, int *__restrict__ agg, const int *__restrict__ rank, int first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn && agg[i] == -1) agg[i] = first + rank[i];
}

__global__ void agg_size_kernel(int nn, const int *__restrict__ agg, int *__restrict__ size) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn && agg[i] >= 0) atomicAdd(size + agg[i], 1);
}

// ---------------------------------------------------------------------------
// prolongator
// ---------------------------------------------------------------------------
__global__ void tentative_kernel(int n, int block, const int *__restrict__ agg, const int *__restrict__ size,
                                 int *__restrict__ tcol, double *__restrict__ tval) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int i = row / block, comp = row % block;
  if (agg[i] >= 0) {
    tcol[row] = agg[i] * block + comp;
    tval[row] = 1.0 / sqrt(static_cast<double>(size[agg[i]]));
  } else {
    tcol[row] = -1;
    tval[row] = 0.0;
  }
}

// Filtered matrix: an entry is kept when its node column is the row's own
// node or a strong neighbour of it; the others are lumped into the diagonal.
// Also the row's Gershgorin ratio of D_F^-1 A_F, max-reduced.
__global__ void filter_kernel(int n, int block, const int *__restrict__ rp, const int *__restrict__ ci,
                              const double *__restrict__ v, const int *__restrict__ nrp,
                              const int *__restrict__ nci, const unsigned char *__restrict__ strong,
                              unsigned char *__restrict__ keep, double *__restrict__ fdiag,
                              unsigned long long *__restrict__ rho_bits) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int i = row / block;
  double lump = 0.0, d = 0.0;
  for (int k = rp[row]; k < rp[row + 1]; ++k) {
    const int j = ci[k] / block;
    bool kp = j == i;
    if (!kp) {
      int lo = nrp[i], hi = nrp[i + 1];  // lower_bound of j
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (nci[mid] < j) lo = mid + 1;
        else hi = mid;
      }
      kp = lo < nrp[i + 1] && nci[lo] == j && strong[lo];
    }
    keep[k] = kp ? 1 : 0;
    if (ci[k] == row) d += v[k];
    else if (!kp) lump += v[k];
  }
  const double fd = d + lump;
  fdiag[row] = fd;
  double s = fabs(fd);
  for (int k = rp[row]; k < rp[row + 1]; ++k)
    if (keep[k] && ci[k] != row) s += fabs(v[k]);
  if (fd != 0.0) atomicMax(rho_bits, static_cast<unsigned long long>(__double_as_longlong(s / fabs(fd))));
}

// P = (I - omega D_F^-1 A_F) P_tent, one row per thread: the distinct
// prolongator columns collect in a scratch run at the row's own offset in A,
// summed in entry order, then sorted by column.
__global__ void prolong_rows_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                    const double *__restrict__ v, const unsigned char *__restrict__ keep,
                                    const double *__restrict__ fdiag, const int *__restrict__ tcol,
                                    const double *__restrict__ tval, double omega, int *__restrict__ pcnt,
                                    int *__restrict__ scol, double *__restrict__ sval) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int base = rp[row];
  const double fd = fdiag[row];
  const double scale = fd != 0.0 ? omega / fd : 0.0;
  int m = 0;
  for (int k = rp[row]; k < rp[row + 1]; ++k) {
    if (!keep[k]) continue;
    const int c = ci[k];
    if (tcol[c] < 0) continue;
    const double afv = c == row ? fd : v[k];
    const double coef = (c == row ? 1.0 : 0.0) - scale * afv;
    const int pc = tcol[c];
    const double add = coef * tval[c];
    int t = 0;
    while (t < m && scol[base + t] != pc) ++t;
    if (t == m) {
      scol[base + m] = pc;
      sval[base + m] = 0.0 + add;
      ++m;
    } else {
      sval[base + t] += add;
    }
  }
  for (int a = 1; a < m; ++a) {  // insertion sort by column (columns are distinct)
    const int kc = scol[base + a];
    const double kv = sval[base + a];
    int b = a - 1;
    while (b >= 0 && scol[base + b] > kc) {
      scol[base + b + 1] = scol[base + b];
      sval[base + b + 1] = sval[base + b];
      --b;
    }
    scol[base + b + 1] = kc;
    sval[base + b + 1] = kv;
  }
  pcnt[row] = m;
}

__global__ void compact_rows_kernel(int n, const int *__restrict__ src_rp, const int *__restrict__ dst_rp,
                                    const int *__restrict__ scol, const double *__restrict__ sval,
                                    int *__restrict__ dci, double *__restrict__ dv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int s0 = src_rp[row], d0 = dst_rp[row], m = dst_rp[row + 1] - d0;
  for (int t = 0; t < m; ++t) {
    dci[d0 + t] = scol[s0 + t];
    dv[d0 + t] = sval[s0 + t];
  }
}

// ---------------------------------------------------------------------------
// transpose: R = P^T, entries of each R row in increasing P-row order
// ---------------------------------------------------------------------------
__global__ void col_count_kernel(int nnz, const int *__restrict__ ci, int *__restrict__ cnt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) atomicAdd(cnt + ci[k], 1);
}

__global__ void transpose_fill_kernel(int rows, const int *__restrict__ rp, const int *__restrict__ ci,
                                      const double *__restrict__ v, const int *__restrict__ trp,
                                      int *__restrict__ cursor, int *__restrict__ tci, double *__restrict__ tv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  for (int k = rp[row]; k < rp[row + 1]; ++k) {
    const int c = ci[k];
    const int pos = trp[c] + atomicAdd(cursor + c, 1);
    tci[pos] = row;
    tv[pos] = v[k];
  }
}

__global__ void segment_sort_kernel(int nseg, const int *__restrict__ rp, int *__restrict__ ci,
                                    double *__restrict__ v) {
  const int sgm = blockIdx.x * blockDim.x + threadIdx.x;
  if (sgm >= nseg) return;
  const int b0 = rp[sgm], b1 = rp[sgm + 1];
  for (int a = b0 + 1; a < b1; ++a) {
    const int kc = ci[a];
    const double kv = v[a];
    int b = a - 1;
    while (b >= b0 && ci[b] > kc) {
      ci[b + 1] = ci[b];
      v[b + 1] = v[b];
      --b;
    }
    ci[b + 1] = kc;
    v[b + 1] = kv;
  }
}

// ---------------------------------------------------------------------------
// C = A B, one warp per row of C
// ---------------------------------------------------------------------------
constexpr int kHashCap = 1024;        // slots per warp (power of two)
constexpr int kSpgemmWarps = 4;       // warps per block: 4 * 12 KB of shared memory
constexpr int kSpgemmSmem = kSpgemmWarps * kHashCap * (sizeof(int) + sizeof(double));

__device__ __forceinline__ int hash_slot(int key) {
  return static_cast<int>((static_cast<uint32_t>(key) * 2654435761u) >> 22) & (kHashCap - 1);
}

// Count pass (kFill false): cnt[row] = distinct columns of the row. Fill
// pass: the row's entries at crp[row], sorted by column. In one round the
// lanes hold distinct columns (one row of B), so each slot has one writer
// per round, and rounds follow the host's product order.
template <bool kFill>
__global__ void __launch_bounds__(32 * kSpgemmWarps) spgemm_kernel(
    int rows, const int *__restrict__ arp, const int *__restrict__ aci, const double *__restrict__ av,
    const int *__restrict__ brp, const int *__restrict__ bci, const double *__restrict__ bv,
    int *__restrict__ cnt, const int *__restrict__ crp, int *__restrict__ cci, double *__restrict__ cv,
    int *__restrict__ overflow) {
  extern __shared__ __align__(16) unsigned char spgemm_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *vals = reinterpret_cast<double *>(spgemm_smem) + warp * kHashCap;
  int *keys = reinterpret_cast<int *>(spgemm_smem + kSpgemmWarps * kHashCap * sizeof(double)) + warp * kHashCap;
  for (int row = blockIdx.x * kSpgemmWarps + warp; row < rows; row += gridDim.x * kSpgemmWarps) {
    for (int t = lane; t < kHashCap; t += 32) {
      keys[t] = -1;
      vals[t] = 0.0;
    }
    __syncwarp();
    int distinct = 0;
    bool full = false;
    for (int k = arp[row]; k < arp[row + 1]; ++k) {
      const int j = aci[k];
      const double a = av[k];
      const int q1 = brp[j + 1];
      for (int q0 = brp[j]; q0 < q1; q0 += 32) {
        const int q = q0 + lane;
        if (q < q1 && !full) {
          const int col = bci[q];
          int slot = hash_slot(col), probes = 0;
          for (;;) {
            const int prev = atomicCAS(keys + slot, -1, col);
            if (prev == -1) {
              ++distinct;
              break;
            }
            if (prev == col) break;
            slot = (slot + 1) & (kHashCap - 1);
            if (++probes == kHashCap) {
              full = true;
              break;
            }
          }
          if (kFill && !full) vals[slot] += a * bv[q];
        }
        __syncwarp();
      }
    }
    if (__any_sync(0xffffffffu, full)) {
      if (lane == 0) atomicExch(overflow, 1);
      continue;
    }
    if (!kFill) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) distinct += __shfl_xor_sync(0xffffffffu, distinct, o);
      if (lane == 0) cnt[row] = distinct;
      continue;
    }
    // compact the used slots to the front, chunk by chunk (a slot only moves
    // towards lower indices, after its chunk has been read)
    int m = 0;
    for (int c0 = 0; c0 < kHashCap; c0 += 32) {
      const int key = keys[c0 + lane];
      const double val = vals[c0 + lane];
      const unsigned used = __ballot_sync(0xffffffffu, key != -1);
      __syncwarp();
      if (key != -1) {
        const int pos = m + __popc(used & ((1u << lane) - 1));
        keys[pos] = key;
        vals[pos] = val;
      }
      m += __popc(used);
      __syncwarp();
    }
    int p2 = 32;
    while (p2 < m) p2 <<= 1;
    for (int t = m + lane; t < p2; t += 32) keys[t] = INT_MAX;
    __syncwarp();
    // bitonic sort of keys[0..p2) with their values
    for (int size = 2; size <= p2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = lane; t < p2 / 2; t += 32) {
          const int lo = 2 * stride * (t / stride) + (t % stride), hi = lo + stride;
          const bool up = (lo & size) == 0;
          const int kl = keys[lo], kh = keys[hi];
          if ((kl > kh) == up) {
            keys[lo] = kh;
            keys[hi] = kl;
            const double vl = vals[lo];
            vals[lo] = vals[hi];
            vals[hi] = vl;
          }
        }
        __syncwarp();
      }
    }
    const int c0 = crp[row];
    for (int t = lane; t < m; t += 32) {
      cci[c0 + t] = keys[t];
      cv[c0 + t] = vals[t];
    }
    __syncwarp();
  }
}

void check_overflow(const DBuf<int> &overflow, cudaStream_t s) {
  int of = 0;
  SCK(cudaMemcpyAsync(&of, overflow.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  if (of != 0) throw std::runtime_error("GPU setup: a row of a Galerkin product has more than 1024 columns");
}

DCsr spgemm_device(const DCsr &a, const DCsr &b, cudaStream_t s, DBuf<int> &overflow) {
  DCsr c;
  c.rows = a.rows;
  c.cols = b.cols;
  DBuf<int> cnt(static_cast<size_t>(a.rows) + 1, s);
  const int grid = std::max(1, std::min((a.rows + kSpgemmWarps - 1) / kSpgemmWarps, 148 * 64));
  SCK(cudaMemsetAsync(overflow.get(), 0, sizeof(int), s));
  spgemm_kernel<false><<<grid, 32 * kSpgemmWarps, kSpgemmSmem, s>>>(a.rows, a.rp.get(), a.ci.get(), a.v.get(),
                                                                    b.rp.get(), b.ci.get(), b.v.get(), cnt.get(),
                                                                    nullptr, nullptr, nullptr, overflow.get());
  check_launch("sparse product (count)");
  c.rp.alloc(static_cast<size_t>(a.rows) + 1, s);
  c.nnz = scan_total(cnt.get(), c.rp.get(), a.rows, s);
  check_overflow(overflow, s);
  c.ci.alloc(c.nnz, s);
  c.v.alloc(c.nnz, s);
  spgemm_kernel<true><<<grid, 32 * kSpgemmWarps, kSpgemmSmem, s>>>(a.rows, a.rp.get(), a.ci.get(), a.v.get(),
                                                                   b.rp.get(), b.ci.get(), b.v.get(), nullptr,
                                                                   c.rp.get(), c.ci.get(), c.v.get(), overflow.get());
  check_launch("sparse product (fill)");
  check_overflow(overflow, s);
  return c;
}

DCsr transpose_device(const DCsr &p, cudaStream_t s) {
  DCsr r;
  r.rows = p.cols;
  r.cols = p.rows;
  r.nnz = p.nnz;
  DBuf<int> cnt(static_cast<size_t>(p.cols) + 1, s), cursor(static_cast<size_t>(p.cols) + 1, s);
  SCK(cudaMemsetAsync(cnt.get(), 0, sizeof(int) * (static_cast<size_t>(p.cols) + 1), s));
  SCK(cudaMemsetAsync(cursor.get(), 0, sizeof(int) * (static_cast<size_t>(p.cols) + 1), s));
  col_count_kernel<<<grid_for(p.nnz), 256, 0, s>>>(p.nnz, p.ci.get(), cnt.get());
  check_launch("transpose count");
  r.rp.alloc(static_cast<size_t>(p.cols) + 1, s);
  scan_into(cnt.get(), r.rp.get(), p.cols, s);
  r.ci.alloc(p.nnz, s);
  r.v.alloc(p.nnz, s);
  transpose_fill_kernel<<<grid_for(p.rows), 256, 0, s>>>(p.rows, p.rp.get(), p.ci.get(), p.v.get(), r.rp.get(),
                                                          cursor.get(), r.ci.get(), r.v.get());
  check_launch("transpose fill");
  segment_sort_kernel<<<grid_for(p.cols), 256, 0, s>>>(p.cols, r.rp.get(), r.ci.get(), r.v.get());
  check_launch("transpose sort");
  return r;
}

// One coarsening step on the device (sa_coarsen with aggregation 1).
struct Step {
  DCsr P, R, Ac;
  DBuf<int> agg;
  int nagg = 0;
  int rounds = 0;
};

Step coarsen_device(const DCsr &A, int block, double eps, cudaStream_t s) {
  const int n = A.rows, nn = n / block;
  Step out;
  // node couplings
  DBuf<int> ncnt(static_cast<size_t>(nn) + 1, s), nrp(static_cast<size_t>(nn) + 1, s);
  couplings_kernel<<<grid_for(nn), 256, 0, s>>>(nn, block, A.rp.get(), A.ci.get(), A.v.get(), ncnt.get(), nullptr,
                                                nullptr, nullptr, nullptr);
  check_launch("node couplings (count)");
  const int ncoup = scan_total(ncnt.get(), nrp.get(), nn, s);
  DBuf<int> nci(ncoup, s);
  DBuf<double> nw(ncoup, s), nd(nn, s);
  couplings_kernel<<<grid_for(nn), 256, 0, s>>>(nn, block, A.rp.get(), A.ci.get(), A.v.get(), nullptr, nrp.get(),
                                                nci.get(), nw.get(), nd.get());
  check_launch("node couplings");
  DBuf<unsigned char> strong(ncoup, s);
  DBuf<int> nstrong(nn, s);
  strength_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nrp.get(), nci.get(), nw.get(), nd.get(), eps * eps,
                                               strong.get(), nstrong.get());
  check_launch("strength");

  // independent set
  DBuf<unsigned char> state(nn, s);
  DBuf<uint64_t> t1(nn, s), t2(nn, s);
  DBuf<int> counter(1, s);
  SCK(cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
  mis_init_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nstrong.get(), state.get(), counter.get());
  check_launch("independent set init");
  int undecided = 0;
  SCK(cudaMemcpyAsync(&undecided, counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  while (undecided > 0) {
    if (++out.rounds > 10000) throw std::runtime_error("GPU setup: independent set did not converge");
    mis_max_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nrp.get(), nci.get(), strong.get(), state.get(), nullptr,
                                                t1.get());
    mis_max_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nrp.get(), nci.get(), strong.get(), state.get(), t1.get(),
                                                t2.get());
    SCK(cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
    mis_decide_kernel<<<grid_for(nn), 256, 0, s>>>(nn, state.get(), t2.get(), counter.get());
    check_launch("independent set round");
    SCK(cudaMemcpyAsync(&undecided, counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
  }

  // aggregates
  DBuf<int> flag(static_cast<size_t>(nn) + 1, s), rid(static_cast<size_t>(nn) + 1, s);
  state_flag_kernel<<<grid_for(nn), 256, 0, s>>>(nn, state.get(), 2, flag.get());
  check_launch("root flags");
  const int nroots = scan_total(flag.get(), rid.get(), nn, s);
  out.agg.alloc(nn, s);
  DBuf<int> claim(nn, s), agg1(nn, s);
  agg_init_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nstrong.get(), state.get(), rid.get(), out.agg.get(),
                                               claim.get());
  claim_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nrp.get(), nci.get(), strong.get(), state.get(), out.agg.get(),
                                            claim.get());
  claim_apply_kernel<<<grid_for(nn), 256, 0, s>>>(nn, out.agg.get(), claim.get());
  check_launch("root neighbourhoods");
  SCK(cudaMemcpyAsync(agg1.get(), out.agg.get(), sizeof(int) * nn, cudaMemcpyDeviceToDevice, s));
  join_kernel<<<grid_for(nn), 256, 0, s>>>(nn, nrp.get(), nci.get(), nw.get(), strong.get(), agg1.get(),
                                           out.agg.get());
  free_flag_kernel<<<grid_for(nn), 256, 0, s>>>(nn, out.agg.get(), flag.get());
  check_launch("join");
  const int nleft = scan_total(flag.get(), rid.get(), nn, s);
  singleton_kernel<<<grid_for(nn), 256, 0, s>>>(nn, out.agg.get(), rid.get(), nroots);
  check_launch("singletons");
  out.nagg = nroots + nleft;
  if (out.nagg == 0) return out;

  // tentative prolongator
  const int nc = out.nagg * block;
  DBuf<int> size(out.nagg, s), tcol(n, s);
  DBuf<double> tval(n, s);
  SCK(cudaMemsetAsync(size.get(), 0, sizeof(int) * out.nagg, s));
  agg_size_kernel<<<grid_for(nn), 256, 0, s>>>(nn, out.agg.get(), size.get());
  tentative_kernel<<<grid_for(n), 256, 0, s>>>(n, block, out.agg.get(), size.get(), tcol.get(), tval.get());
  check_launch("tentative prolongator");

  // filtered diagonal, damping
  DBuf<unsigned char> keep(A.nnz, s);
  DBuf<double> fdiag(n, s);
  DBuf<unsigned long long> rho_bits(1, s);
  SCK(cudaMemsetAsync(rho_bits.get(), 0, sizeof(unsigned long long), s));
  filter_kernel<<<grid_for(n), 256, 0, s>>>(n, block, A.rp.get(), A.ci.get(), A.v.get(), nrp.get(), nci.get(),
                                            strong.get(), keep.get(), fdiag.get(), rho_bits.get());
  check_launch("filtered matrix");
  unsigned long long rb = 0;
  SCK(cudaMemcpyAsync(&rb, rho_bits.get(), sizeof(rb), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  double rho = 0.0;
  static_assert(sizeof(rho) == sizeof(rb), "double is 64 bits");
  std::memcpy(&rho, &rb, sizeof(rho));
  const double omega = rho > 0.0 ? (4.0 / 3.0) / rho : 0.0;

  // smoothed prolongator
  DBuf<int> pcnt(static_cast<size_t>(n) + 1, s), scol(A.nnz, s);
  DBuf<double> sval(A.nnz, s);
  prolong_rows_kernel<<<grid_for(n), 256, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), keep.get(), fdiag.get(),
                                                  tcol.get(), tval.get(), omega, pcnt.get(), scol.get(),
                                                  sval.get());
  check_launch("prolongator rows");
  out.P.rows = n;
  out.P.cols = nc;
  out.P.rp.alloc(static_cast<size_t>(n) + 1, s);
  out.P.nnz = scan_total(pcnt.get(), out.P.rp.get(), n, s);
  out.P.ci.alloc(out.P.nnz, s);
  out.P.v.alloc(out.P.nnz, s);
  compact_rows_kernel<<<grid_for(n), 256, 0, s>>>(n, A.rp.get(), out.P.rp.get(), scol.get(), sval.get(),
                                                  out.P.ci.get(), out.P.v.get());
  check_launch("prolongator");

  // R = P^T, Ac = R (A P)
  out.R = transpose_device(out.P, s);
  DBuf<int> overflow(1, s);
  const DCsr AP = spgemm_device(A, out.P, s, overflow);
  out.Ac = spgemm_device(out.R, AP, s, overflow);
  SCK(cudaStreamSynchronize(s));
  return out;
}

Csr download(const DCsr &d, cudaStream_t s) {
  Csr h;
  h.rows = d.rows;
  h.cols = d.cols;
  h.rp.resize(static_cast<size_t>(d.rows) + 1);
  h.ci.resize(d.nnz);
  h.v.resize(d.nnz);
  SCK(cudaMemcpyAsync(h.rp.data(), d.rp.get(), sizeof(int) * h.rp.size(), cudaMemcpyDeviceToHost, s));
  if (d.nnz > 0) {
    SCK(cudaMemcpyAsync(h.ci.data(), d.ci.get(), sizeof(int) * h.ci.size(), cudaMemcpyDeviceToHost, s));
    SCK(cudaMemcpyAsync(h.v.data(), d.v.get(), sizeof(double) * h.v.size(), cudaMemcpyDeviceToHost, s));
  }
  return h;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

bool rows_sorted_unique(const Csr &a) {
  for (int r = 0; r < a.rows; ++r)
    for (int k = a.rp[r] + 1; k < a.rp[r + 1]; ++k)
      if (a.ci[k] <= a.ci[k - 1]) return false;
  return true;
}

namespace {

DCsr upload_csr(const Csr &a, cudaStream_t s) {
  DCsr d;
  d.rows = a.rows;
  d.cols = a.cols;
  d.nnz = a.nnz();
  d.rp.alloc(a.rp.size(), s);
  d.ci.alloc(d.nnz, s);
  d.v.alloc(d.nnz, s);
  SCK(cudaMemcpyAsync(d.rp.get(), a.rp.data(), sizeof(int) * a.rp.size(), cudaMemcpyHostToDevice, s));
  if (d.nnz > 0) {
    SCK(cudaMemcpyAsync(d.ci.get(), a.ci.data(), sizeof(int) * d.nnz, cudaMemcpyHostToDevice, s));
    SCK(cudaMemcpyAsync(d.v.get(), a.v.data(), sizeof(double) * d.nnz, cudaMemcpyHostToDevice, s));
  }
  return d;
}

}  // namespace

std::vector<Csr> galerkin_device(const Csr &a0, const std::vector<Csr> &P, const std::vector<Csr> &R, int levels,
                                 int device) {
  if (levels < 1 || static_cast<int>(P.size()) < levels - 1 || static_cast<int>(R.size()) < levels - 1)
    throw std::runtime_error("Galerkin refresh: transfer operators missing");
  for (int k = 0; k + 1 < levels; ++k)
    if (!rows_sorted_unique(P[k]) || !rows_sorted_unique(R[k]))
      throw std::runtime_error("Galerkin refresh: transfer rows must be sorted and duplicate-free");
  if (!rows_sorted_unique(a0)) throw std::runtime_error("Galerkin refresh: matrix rows must be sorted and duplicate-free");
  SCK(cudaSetDevice(device));
  cudaStream_t s = nullptr;
  SCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  std::vector<Csr> out;
  out.push_back(a0);
  try {
    SCK(cudaFuncSetAttribute(spgemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpgemmSmem));
    SCK(cudaFuncSetAttribute(spgemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpgemmSmem));
    DBuf<int> overflow(1, s);
    DCsr cur = upload_csr(a0, s);
    for (int k = 0; k + 1 < levels; ++k) {
      const DCsr dp = upload_csr(P[k], s), dr = upload_csr(R[k], s);
      const DCsr ap = spgemm_device(cur, dp, s, overflow);
      DCsr ac = spgemm_device(dr, ap, s, overflow);
      out.push_back(download(ac, s));
      SCK(cudaStreamSynchronize(s));
      cur = std::move(ac);
    }
    SCK(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    throw;
  }
  SCK(cudaStreamDestroy(s));
  return out;
}

Hierarchy build_hierarchy_device(const Csr &a, const SaOptions &opt, int device, DeviceSetupStats *stats) {
  const auto t0 = std::chrono::steady_clock::now();
  a.check("AMGHierarchyBuilder input");
  if (a.rows != a.cols) throw std::runtime_error("AMGHierarchyBuilder: matrix must be square.");
  if (opt.max_levels <= 0) throw std::runtime_error("AMGHierarchyBuilder: maxLevels must be positive.");
  if (opt.min_dofs <= 0) throw std::runtime_error("AMGHierarchyBuilder: minDofs must be positive.");
  if (opt.block <= 0 || opt.block > kMaxBlock) throw std::runtime_error("GPU setup: block size must be 1..8");
  if (a.rows % opt.block != 0)
    throw std::runtime_error("SmoothedAggregationCoarsener: matrix size is not divisible by block size.");
  if (!rows_sorted_unique(a))
    throw std::runtime_error("GPU setup: every row needs sorted, duplicate-free column indices");
  SCK(cudaSetDevice(device));
  cudaStream_t s = nullptr;
  SCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  DeviceSetupStats st;
  Hierarchy h;
  h.block = opt.block;
  try {
    SCK(cudaFuncSetAttribute(spgemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpgemmSmem));
    SCK(cudaFuncSetAttribute(spgemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpgemmSmem));
    auto tu = std::chrono::steady_clock::now();
    DCsr cur;
    cur.rows = a.rows;
    cur.cols = a.cols;
    cur.nnz = a.nnz();
    cur.rp.alloc(a.rp.size(), s);
    cur.ci.alloc(cur.nnz, s);
    cur.v.alloc(cur.nnz, s);
    SCK(cudaMemcpyAsync(cur.rp.get(), a.rp.data(), sizeof(int) * a.rp.size(), cudaMemcpyHostToDevice, s));
    if (cur.nnz > 0) {
      SCK(cudaMemcpyAsync(cur.ci.get(), a.ci.data(), sizeof(int) * cur.nnz, cudaMemcpyHostToDevice, s));
      SCK(cudaMemcpyAsync(cur.v.get(), a.v.data(), sizeof(double) * cur.nnz, cudaMemcpyHostToDevice, s));
    }
    SCK(cudaStreamSynchronize(s));
    st.upload_ms = ms_since(tu);
    h.A.push_back(a);
    for (int level = 0; level < opt.max_levels; ++level) {
      if (cur.rows <= opt.min_dofs) break;
      auto tb = std::chrono::steady_clock::now();
      Step step = coarsen_device(cur, opt.block, opt.eps_strong * std::ldexp(1.0, -level), s);
      SCK(cudaStreamSynchronize(s));
      st.build_ms += ms_since(tb);
      st.mis_rounds += step.rounds;
      if (step.nagg == 0 || step.Ac.rows == 0 || step.Ac.rows >= cur.rows) break;
      auto td = std::chrono::steady_clock::now();
      std::vector<int> agg(cur.rows / opt.block);
      SCK(cudaMemcpyAsync(agg.data(), step.agg.get(), sizeof(int) * agg.size(), cudaMemcpyDeviceToHost, s));
      h.P.push_back(download(step.P, s));
      h.R.push_back(download(step.R, s));
      h.A.push_back(download(step.Ac, s));
      SCK(cudaStreamSynchronize(s));
      h.agg.push_back(std::move(agg));
      st.download_ms += ms_since(td);
      cur = std::move(step.Ac);
    }
    cur = DCsr();
    SCK(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    throw;
  }
  SCK(cudaStreamDestroy(s));
  st.total_ms = ms_since(t0);
  if (stats != nullptr) *stats = st;
  return h;
}

}  // namespace gsb
