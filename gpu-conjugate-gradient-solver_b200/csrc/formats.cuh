// Device-side matrix formats shared by the solvers: the SELL-32 and
// CSR-vector builders and uploads, a device-memory arena owned by one solver,
// and the dense inverse used for the coarsest level. Host code only.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <utility>
#include <vector>

#include "kernels.cuh"
#include "setup.h"
#include "solver.h"

#define GSB_CK(x) ::gsb::cuda_check((x), #x)

namespace gsb {

// ---------------------------------------------------------------------------
// device memory owned by one solver
// ---------------------------------------------------------------------------
class Arena {
 public:
  ~Arena() {
    for (void *p : ptrs_) cudaFree(p);
  }
  template <typename T>
  T *alloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    GSB_CK(cudaMalloc(&p, n * sizeof(T)));
    ptrs_.push_back(p);
    bytes_ += n * sizeof(T);
    return static_cast<T *>(p);
  }
  template <typename T>
  T *upload(const std::vector<T> &h) {
    T *d = alloc<T>(h.size());
    if (!h.empty()) GSB_CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  size_t bytes() const { return bytes_; }

 private:
  std::vector<void *> ptrs_;
  size_t bytes_ = 0;
};

// ---------------------------------------------------------------------------
// host construction of SELL-32 / BELL-32
// ---------------------------------------------------------------------------
template <typename T>
struct HostSell {
  int rows = 0, cols = 0, g = 1;
  std::vector<int> srow, sptr, col;
  std::vector<T> val, diag;
};

// Slices of at most 32 / g rows that never cross an entry of `bounds`
// (ascending, starting at 0 and ending at a.rows). With g lanes per row the
// k-th stored entry of local row i goes to lane i * g + k % g as that lane's
// slot k / g; slots keep the slot-pair interleave of SELL-32.
template <typename T>
HostSell<T> make_sell(const Csr &a, const std::vector<int> &bounds, bool split_diag, int g = 1) {
  if (g != 1 && g != 2 && g != 4 && g != 8) throw std::runtime_error("SELL: lanes per row must be 1, 2, 4 or 8");
  HostSell<T> h;
  h.rows = a.rows;
  h.cols = a.cols;
  h.g = g;
  const int per = 32 / g;
  for (size_t b = 0; b + 1 < bounds.size(); ++b)
    for (int r = bounds[b]; r < bounds[b + 1]; r += per) h.srow.push_back(r);
  h.srow.push_back(a.rows);
  const int ns = static_cast<int>(h.srow.size()) - 1;
  std::vector<int> width(ns, 0);  // slots per lane, even
  parallel_for(ns, [&](long long s0, long long s1) {
    for (long long s = s0; s < s1; ++s) {
      int w = 0;
      for (int r = h.srow[s]; r < h.srow[s + 1]; ++r) {
        int c = 0;
        for (int k = a.rp[r]; k < a.rp[r + 1]; ++k)
          if (!(split_diag && a.ci[k] == r)) ++c;
        w = std::max(w, (c + g - 1) / g);
      }
      width[s] = (w + 1) & ~1;
    }
  }, 256);
  h.sptr.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s) {
    if (static_cast<long long>(h.sptr[s]) + 32LL * width[s] > 2147483647LL)
      throw std::runtime_error("SELL: too many stored entries for 32-bit offsets");
    h.sptr[s + 1] = h.sptr[s] + 32 * width[s];
  }
  h.col.assign(h.sptr[ns], 0);
  h.val.assign(h.sptr[ns], T(0));
  if (split_diag) h.diag.assign(a.rows, T(0));
  parallel_for(ns, [&](long long s0, long long s1) {
    for (long long s = s0; s < s1; ++s) {
      // Padding gathers x[pad] * 0. Square level matrices pad with the slice's
      // own first row (same colour: skipped by a zero-guess sweep); transfer
      // operators with a column the slice really uses, so that in a
      // block-diagonal batch the padding never reads another system's vector.
      int pad = std::min(h.srow[s], a.cols - 1);
      if (!split_diag)
        for (int r = h.srow[s]; r < h.srow[s + 1]; ++r)
          if (a.rp[r + 1] > a.rp[r]) {
            pad = a.ci[a.rp[r]];
            break;
          }
      for (int p = h.sptr[s]; p < h.sptr[s + 1]; ++p) h.col[p] = pad;
      for (int r = h.srow[s]; r < h.srow[s + 1]; ++r) {
        const int local = r - h.srow[s];
        int k = 0;
        for (int e = a.rp[r]; e < a.rp[r + 1]; ++e) {
          if (split_diag && a.ci[e] == r) {
            h.diag[r] = T(a.v[e]);
            continue;
          }
          const int lane = local * g + k % g, kk = k / g;
          const int idx = h.sptr[s] + (kk >> 1) * 64 + 2 * lane + (kk & 1);
          h.col[idx] = a.ci[e];
          h.val[idx] = T(a.v[e]);
          ++k;
        }
      }
    }
  }, 256);
  return h;
}

template <typename T>
struct DevSell {
  int rows = 0, cols = 0, nslices = 0, g = 1;
  long long stored = 0;
  int *srow = nullptr, *sptr = nullptr, *col = nullptr;
  T *val = nullptr, *diag = nullptr;
  std::vector<int> h_srow;  // slice -> first row, kept on the host for launch ranges
  SellView<T> view() const { return SellView<T>{rows, cols, nslices, srow, sptr, col, val, diag}; }
};

template <typename T>
DevSell<T> upload_sell(Arena &ar, const HostSell<T> &h) {
  DevSell<T> d;
  d.rows = h.rows;
  d.cols = h.cols;
  d.g = h.g;
  d.nslices = static_cast<int>(h.srow.size()) - 1;
  d.stored = h.sptr.back();
  d.srow = ar.upload(h.srow);
  d.sptr = ar.upload(h.sptr);
  d.col = ar.upload(h.col);
  d.val = ar.upload(h.val);
  d.diag = h.diag.empty() ? nullptr : ar.upload(h.diag);
  d.h_srow = h.srow;
  return d;
}

template <typename T>
struct DevCsrv {
  int rows = 0;
  int *rp = nullptr, *ci = nullptr;
  T *v = nullptr, *diag = nullptr;
  CsrvView<T> view() const { return CsrvView<T>{rows, rp, ci, v, diag}; }
};

// CSR with the diagonal split off (square level matrices) or kept (transfer
// operators), columns in stored order.
template <typename T>
DevCsrv<T> upload_csrv(Arena &ar, const Csr &a, bool split_diag) {
  std::vector<int> rp(a.rows + 1, 0);
  std::vector<T> diag;
  if (split_diag) diag.assign(a.rows, T(0));
  for (int r = 0; r < a.rows; ++r) {
    int c = a.rp[r + 1] - a.rp[r];
    if (split_diag)
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) c -= a.ci[k] == r ? 1 : 0;
    rp[r + 1] = rp[r] + c;
  }
  std::vector<int> ci(rp[a.rows]);
  std::vector<T> v(rp[a.rows]);
  parallel_for(a.rows, [&](long long r0, long long r1) {
    for (long long r = r0; r < r1; ++r) {
      int dst = rp[r];
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
        if (split_diag && a.ci[k] == r) {
          diag[r] = T(a.v[k]);
          continue;
        }
        ci[dst] = a.ci[k];
        v[dst] = T(a.v[k]);
        ++dst;
      }
    }
  }, row_grain(a.rows, a.nnz()));
  DevCsrv<T> d;
  d.rows = a.rows;
  d.rp = ar.upload(rp);
  d.ci = ar.upload(ci);
  d.v = ar.upload(v);
  d.diag = split_diag ? ar.upload(diag) : nullptr;
  return d;
}

// Coarsest levels up to this many rows are inverted on the host (below), larger
// ones on the GPU (spd_inverse_device).
constexpr int kHostInverseRows = 1000;

// Dense inverse of an SPD matrix through its Cholesky factor, A^-1 = L^-T L^-1.
inline std::vector<double> cholesky_inverse(const Csr &a) {
  const int n = a.rows;
  std::vector<double> m(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) m[static_cast<size_t>(i) * n + a.ci[k]] += a.v[k];
  // in-place lower Cholesky
  for (int j = 0; j < n; ++j) {
    double d = m[static_cast<size_t>(j) * n + j];
    for (int k = 0; k < j; ++k) d -= m[static_cast<size_t>(j) * n + k] * m[static_cast<size_t>(j) * n + k];
    if (!(d > 0.0)) throw std::runtime_error("coarsest level matrix is not SPD (Cholesky failed)");
    const double ljj = std::sqrt(d);
    m[static_cast<size_t>(j) * n + j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = m[static_cast<size_t>(i) * n + j];
      const double *li = &m[static_cast<size_t>(i) * n];
      const double *lj = &m[static_cast<size_t>(j) * n];
      for (int k = 0; k < j; ++k) s -= li[k] * lj[k];
      m[static_cast<size_t>(i) * n + j] = s / ljj;
    }
  }
  // W = L^-1 (lower triangular), column by column
  std::vector<double> w(static_cast<size_t>(n) * n, 0.0);
  for (int c = 0; c < n; ++c) {
    for (int i = c; i < n; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) s -= m[static_cast<size_t>(i) * n + k] * w[static_cast<size_t>(k) * n + c];
      w[static_cast<size_t>(i) * n + c] = s / m[static_cast<size_t>(i) * n + i];
    }
  }
  // A^-1 = W^T W
  std::vector<double> inv(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += w[static_cast<size_t>(k) * n + i] * w[static_cast<size_t>(k) * n + j];
      inv[static_cast<size_t>(i) * n + j] = s;
      inv[static_cast<size_t>(j) * n + i] = s;
    }
  return inv;
}

inline int sm_count(int device) {
  int v = 0;
  GSB_CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
  return v;
}

// Launches a V-cycle kernel (256 threads per block) on stream s. With
// `overlap` the launch carries programmatic stream serialization: its CTAs may
// become resident while the previous kernel in the stream drains, and the
// kernel's pass_entry holds them until that kernel's writes are visible. Under
// stream capture this becomes a programmatic edge of the CUDA graph.
template <typename... P, typename... A>
void launch_pass(bool overlap, void (*kernel)(P...), int grid, cudaStream_t s, A &&...args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(grid));
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = overlap ? attr : nullptr;
  cfg.numAttrs = overlap ? 1 : 0;
  GSB_CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

inline int blocks_for(long long threads, int cap) {
  long long b = (threads + 255) / 256;
  if (b < 1) b = 1;
  return static_cast<int>(std::min<long long>(b, cap));
}

}  // namespace gsb
