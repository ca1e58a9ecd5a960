// AMG-PCG solver: hierarchy upload in colour-contiguous order, V-cycle
// launch sequence, and the outer CG loop (host-checked, or CUDA-graph
// replayed with a device-side stop flag).
//
// Ordering. For every level k the reference permutes A_k by the caller's
// permutation pi_k (permuteMatrix, src/Smoothers/MultigridSmoother.cc:56-66),
// colours the permuted matrix greedily
// (src/Smoothers/SymmetricGaussSeidelSmoother.cc:33-43) and sweeps colour by
// colour through the list of vertices grouped by colour. Here the level is
// stored directly in that grouped order (internal index = position in the
// colour-grouped vertex list), so a colour pass touches a contiguous row
// range and reads the matrix with coalesced loads. The same relabelling is
// applied to P and R and, at level 0, to the CG vectors; results are mapped
// back to the caller's order at the end of the solve.
#include "solver.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <mutex>
#include <type_traits>
#include <numeric>
#include <unordered_map>

#include "amg_setup.h"
#include "dense.h"
#include "dense_mma.cuh"
#include "formats.cuh"
#include "kernels.cuh"
#include "staged.cuh"
#include "sweep.cuh"
#include "tail.cuh"

namespace gsb {

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) cuda_check((x), #x)

// Strength threshold and same-colour mass bound of the coarse levels'
// colouring under coloring 2 (relaxed_coloring in setup.cc).
constexpr double kRelaxedTheta = 0.05;
constexpr double kRelaxedRho = 0.5;
#define CKL(what) (cuda_check(cudaGetLastError(), what), ++launches_)

namespace {

// Shared memory of one bulk-copy staged block pass over BELL-1 slices of at
// most `max_slots` block slots per lane; 0 when it does not fit one block.
template <typename VT>
size_t staged_smem(int max_slots, int device) {
  const size_t bytes = kStagedWarps * staged_warp_bytes<VT>(std::max(1, max_slots));
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  return bytes <= static_cast<size_t>(optin) ? bytes : 0;
}

// Whether a level of `max_slots` block slots per lane can run the staged
// passes; if so, the kernels' dynamic shared memory limit is raised to the
// device's opt-in maximum (a limit only: residency follows the bytes each
// launch asks for). Called outside any stream capture: at tuning, at the
// tune cache's load, or when sweep_launch forces the staged passes.
template <typename VT>
bool prepare_staged(int max_slots, int device) {
  if (staged_smem<VT>(max_slots, device) == 0) return false;
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, VT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, VT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, VT, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          optin));
  if (!std::is_same<VT, double>::value) {
    CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            optin));
    CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            optin));
    CK(cudaFuncSetAttribute(bell_gs_staged_kernel<VT, double, false, true>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  }
  return true;
}

template <typename T>
struct HostBell {
  int nodes = 0, g = 1;
  std::vector<int> srow, bptr, col;
  std::vector<T> val, diag, dinv;
};

template <typename T>
// BELL-32 with g lanes per node (slices of 32 / g nodes): block q of local
// node i goes to lane i * g + q % g as that lane's block slot q / g.
HostBell<T> make_bell(const Csr &a, const std::vector<int> &node_bounds, int g = 1) {
  if (a.rows % 3 != 0) throw std::runtime_error("3x3 block smoother requires number of DOFs divisible by 3.");
  if (g != 1 && g != 2 && g != 4 && g != 8) throw std::runtime_error("BELL: lanes per node must be 1, 2, 4 or 8");
  HostBell<T> h;
  const int nn = a.rows / 3;
  h.nodes = nn;
  h.g = g;
  // block columns of each node row (sorted, unique, diagonal excluded)
  std::vector<std::vector<int>> bcols(nn);
  parallel_for(nn, [&](long long I0, long long I1) {
    for (long long I = I0; I < I1; ++I) {
      auto &bc = bcols[I];
      for (long long r = 3 * I; r < 3 * I + 3; ++r)
        for (int k = a.rp[r]; k < a.rp[r + 1]; ++k)
          if (a.ci[k] / 3 != I) bc.push_back(a.ci[k] / 3);
      std::sort(bc.begin(), bc.end());
      bc.erase(std::unique(bc.begin(), bc.end()), bc.end());
    }
  }, row_grain(nn, a.nnz()));
  for (size_t b = 0; b + 1 < node_bounds.size(); ++b)
    for (int r = node_bounds[b]; r < node_bounds[b + 1]; r += 32 / g) h.srow.push_back(r);
  h.srow.push_back(nn);
  const int ns = static_cast<int>(h.srow.size()) - 1;
  h.bptr.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s) {
    int w = 0;
    for (int I = h.srow[s]; I < h.srow[s + 1]; ++I)
      w = std::max(w, (static_cast<int>(bcols[I].size()) + g - 1) / g);
    h.bptr[s + 1] = h.bptr[s] + 32 * w;
  }
  h.col.assign(h.bptr[ns], 0);
  h.val.assign(9 * static_cast<size_t>(h.bptr[ns]), T(0));
  h.diag.assign(9 * static_cast<size_t>(nn), T(0));
  parallel_for(ns, [&](long long s0, long long s1) {  // slices write disjoint ranges
    for (long long s = s0; s < s1; ++s) {
      for (int p = h.bptr[s]; p < h.bptr[s + 1]; ++p) h.col[p] = h.srow[s];
      for (int I = h.srow[s]; I < h.srow[s + 1]; ++I) {
        const int local = I - h.srow[s];
        const auto &bc = bcols[I];
        for (size_t q = 0; q < bc.size(); ++q)
          h.col[h.bptr[s] + (q / g) * 32 + local * g + q % g] = bc[q];
        for (int r = 0; r < 3; ++r) {
          const int row = 3 * I + r;
          for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
            const int J = a.ci[k] / 3, comp = a.ci[k] % 3;
            if (J == I) {
              h.diag[9 * static_cast<size_t>(I) + 3 * r + comp] = T(a.v[k]);
              continue;
            }
            const int q = static_cast<int>(std::lower_bound(bc.begin(), bc.end(), J) - bc.begin());
            const int lane = local * g + q % g, qq = q / g;
            h.val[9 * static_cast<size_t>(h.bptr[s]) + (static_cast<size_t>(qq) * 9 + 3 * r + comp) * 32 + lane] =
                T(a.v[k]);
          }
        }
      }
    }
  }, 64);
  std::vector<double> dinv;
  const int bad = block_inverses3x3(a, dinv);
  if (bad >= 0) throw std::runtime_error("Block diagonal is not SPD.");
  h.dinv.resize(dinv.size());
  for (size_t i = 0; i < dinv.size(); ++i) h.dinv[i] = T(dinv[i]);
  return h;
}

template <typename T>
struct DevBell {
  int nodes = 0, nslices = 0, g = 1;
  int max_slots = 0;  // block slots per lane of the widest slice
  long long stored = 0;
  int *srow = nullptr, *bptr = nullptr, *col = nullptr;
  T *val = nullptr, *diag = nullptr, *dinv = nullptr;
  std::vector<int> h_srow;
  BellView<T> view() const { return BellView<T>{nodes, nslices, srow, bptr, col, val, diag, dinv}; }
};

template <typename T>
DevBell<T> upload_bell(Arena &ar, const HostBell<T> &h) {
  DevBell<T> d;
  d.nodes = h.nodes;
  d.g = h.g;
  d.nslices = static_cast<int>(h.srow.size()) - 1;
  d.stored = 9LL * h.bptr.back();
  d.srow = ar.upload(h.srow);
  d.bptr = ar.upload(h.bptr);
  d.col = ar.upload(h.col);
  d.val = ar.upload(h.val);
  d.diag = ar.upload(h.diag);
  d.dinv = ar.upload(h.dinv);
  d.h_srow = h.srow;
  for (size_t q = 0; q + 1 < h.bptr.size(); ++q) d.max_slots = std::max(d.max_slots, (h.bptr[q + 1] - h.bptr[q]) / 32);
  return d;
}

template <typename T>
struct DevBsrv {
  int nodes = 0;
  int *rp = nullptr, *bc = nullptr;
  T *v = nullptr, *diag = nullptr, *dinv = nullptr;
  BsrvView<T> view() const { return BsrvView<T>{nodes, rp, bc, v, diag, dinv}; }
};

// Block CSR of the off-diagonal 3x3 blocks (row-major), diagonal blocks and
// their inverses apart; diag / dinv shared with the BELL copy.
template <typename T>
DevBsrv<T> upload_bsrv(Arena &ar, const Csr &a, const DevBell<T> &bell) {
  const int nn = a.rows / 3;
  std::vector<int> rp(nn + 1, 0), bc;
  std::vector<T> v;
  std::vector<int> cols;
  for (int I = 0; I < nn; ++I) {
    cols.clear();
    for (int r = 3 * I; r < 3 * I + 3; ++r)
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k)
        if (a.ci[k] / 3 != I) cols.push_back(a.ci[k] / 3);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const size_t base = v.size();
    v.resize(base + 9 * cols.size(), T(0));
    for (int r = 0; r < 3; ++r)
      for (int k = a.rp[3 * I + r]; k < a.rp[3 * I + r + 1]; ++k) {
        const int J = a.ci[k] / 3;
        if (J == I) continue;
        const size_t q = std::lower_bound(cols.begin(), cols.end(), J) - cols.begin();
        v[base + 9 * q + 3 * r + a.ci[k] % 3] = T(a.v[k]);
      }
    bc.insert(bc.end(), cols.begin(), cols.end());
    rp[I + 1] = static_cast<int>(bc.size());
  }
  DevBsrv<T> d;
  d.nodes = nn;
  d.rp = ar.upload(rp);
  d.bc = ar.upload(bc);
  d.v = ar.upload(v);
  d.diag = bell.diag;
  d.dinv = bell.dinv;
  return d;
}

// Features of the learned relaxation weights, per colour of one level (rows
// of colour c: [block*offs[c], block*offs[c+1]) in the colour order).
void append_colour_features(const Csr &a, const std::vector<int> &offs, int block, int level,
                            int levels, std::vector<float> &out) {
  const int nc = static_cast<int>(offs.size()) - 1;
  for (int c = 0; c < nc; ++c) {
    const int r0 = block * offs[c], r1 = block * offs[c + 1];
    double dd_sum = 0.0, dd_min = 1e300, dmax = 0.0, dmin = 1e300, len = 0.0;
    for (int r = r0; r < r1; ++r) {
      double d = 0.0, off = 0.0;
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
        if (a.ci[k] == r) d = std::fabs(a.v[k]);
        else off += std::fabs(a.v[k]);
      }
      const double dd = std::log10(std::max(d, 1e-300) / std::max(off, 1e-300));
      const double ddc = std::min(2.0, std::max(-2.0, dd));
      dd_sum += ddc;
      dd_min = std::min(dd_min, ddc);
      dmax = std::max(dmax, d);
      dmin = std::min(dmin, std::max(d, 1e-300));
      len += a.rp[r + 1] - a.rp[r];
    }
    const double rows = std::max(1, r1 - r0);
    out.push_back(static_cast<float>(levels > 1 ? double(level) / (levels - 1) : 0.0));
    out.push_back(static_cast<float>(nc > 1 ? double(c) / (nc - 1) : 0.0));
    out.push_back(static_cast<float>(std::log10(1.0 + (r1 - r0)) / 7.0));
    out.push_back(static_cast<float>(dd_sum / rows / 2.0));
    out.push_back(static_cast<float>((r1 > r0 ? dd_min : 0.0) / 2.0));
    out.push_back(static_cast<float>(r1 > r0 ? std::log10(std::max(dmax, 1e-300) / dmin) / 6.0 : 0.0));
    out.push_back(static_cast<float>(len / rows / 64.0));
    out.push_back(static_cast<float>(double(r1 - r0) / std::max(1, a.rows)));
  }
}

// Eight features per node (3x3 block row) of a block level for the learned
// per-block scalings, written in the caller's node order (internal node I of
// caller node i is q[3 i] / 3): level depth, colour position, log10 of the
// block diagonal dominance ||D_I|| / sum_J ||A_IJ|| (Frobenius norms), log10 of
// the contrast max_J ||A_IJ|| / min_J ||A_IJ|| over the off-diagonal blocks,
// the number of off-diagonal blocks, log10 of ||D_I|| against the level's
// mean, log10 of the largest over the smallest diagonal entry of D_I (the
// anisotropy of the node), and the colour's share of the level's nodes (all
// scaled to about [-1, 1]).
void append_node_features(const Csr &a, const std::vector<int> &offs, const std::vector<int> &q, int level,
                          int levels, std::vector<float> &out) {
  const int nn = a.rows / 3, nc = static_cast<int>(offs.size()) - 1;
  std::vector<double> dnorm(nn, 0.0), off_sum(nn, 0.0), bmax(nn, 0.0), bmin(nn, 1e300), aniso(nn, 0.0);
  std::vector<int> nblk(nn, 0);
  parallel_for(nn, [&](long long i0, long long i1) {
    std::vector<double> acc;
    std::vector<int> cols;
    for (long long I = i0; I < i1; ++I) {
      acc.clear();
      cols.clear();
      double dmax = 0.0, dmin = 1e300;
      for (int r = 3 * static_cast<int>(I); r < 3 * static_cast<int>(I) + 3; ++r)
        for (int e = a.rp[r]; e < a.rp[r + 1]; ++e) {
          const int J = a.ci[e] / 3;
          const double sq = a.v[e] * a.v[e];
          if (a.ci[e] == r) dmax = std::max(dmax, std::fabs(a.v[e])), dmin = std::min(dmin, std::fabs(a.v[e]));
          size_t k = 0;
          while (k < cols.size() && cols[k] != J) ++k;
          if (k == cols.size()) cols.push_back(J), acc.push_back(0.0);
          acc[k] += sq;
        }
      for (size_t k = 0; k < cols.size(); ++k) {
        const double f = std::sqrt(acc[k]);
        if (cols[k] == I) {
          dnorm[I] = f;
        } else {
          off_sum[I] += f;
          bmax[I] = std::max(bmax[I], f);
          bmin[I] = std::min(bmin[I], std::max(f, 1e-300));
          ++nblk[I];
        }
      }
      aniso[I] = dmin < 1e300 ? std::log10(std::max(dmax, 1e-300) / std::max(dmin, 1e-300)) : 0.0;
    }
  });
  double mean_log = 0.0;
  for (int I = 0; I < nn; ++I) mean_log += std::log10(std::max(dnorm[I], 1e-300));
  mean_log /= std::max(1, nn);
  std::vector<int> colour(nn, 0);
  for (int c = 0; c < nc; ++c)
    for (int I = offs[c]; I < offs[c + 1]; ++I) colour[I] = c;
  const size_t base = out.size();
  out.resize(base + 8 * static_cast<size_t>(nn));
  for (int i = 0; i < nn; ++i) {
    const int I = q[3 * i] / 3;
    const int c = colour[I];
    const double dd = std::log10(std::max(dnorm[I], 1e-300) / std::max(off_sum[I], 1e-300));
    float *f = &out[base + 8 * static_cast<size_t>(i)];
    f[0] = static_cast<float>(levels > 1 ? double(level) / (levels - 1) : 0.0);
    f[1] = static_cast<float>(nc > 1 ? double(c) / (nc - 1) : 0.0);
    f[2] = static_cast<float>(std::min(2.0, std::max(-2.0, dd)) / 2.0);
    f[3] = static_cast<float>(nblk[I] > 0 ? std::min(1.0, std::log10(bmax[I] / bmin[I]) / 6.0) : 0.0);
    f[4] = static_cast<float>(nblk[I] / 64.0);
    f[5] = static_cast<float>(std::min(1.0, std::max(-1.0, (std::log10(std::max(dnorm[I], 1e-300)) - mean_log) / 3.0)));
    f[6] = static_cast<float>(std::min(1.0, aniso[I] / 3.0));
    f[7] = static_cast<float>(double(offs[c + 1] - offs[c]) / std::max(1, nn));
  }
}

// ---------------------------------------------------------------------------
// in-place value refresh of device matrices (same sparsity)
// ---------------------------------------------------------------------------
template <typename T>
void refresh_sell(const DevSell<T> &d, const Csr &a, const std::vector<int> &bounds, bool split_diag) {
  if (d.val == nullptr) return;
  const HostSell<T> h = make_sell<T>(a, bounds, split_diag, d.g);
  if (h.sptr.back() != d.stored || static_cast<int>(h.srow.size()) - 1 != d.nslices)
    throw std::runtime_error("update_values: the matrix sparsity changed");
  GSB_CK(cudaMemcpy(d.val, h.val.data(), sizeof(T) * h.val.size(), cudaMemcpyHostToDevice));
  if (split_diag && d.diag != nullptr)
    GSB_CK(cudaMemcpy(d.diag, h.diag.data(), sizeof(T) * h.diag.size(), cudaMemcpyHostToDevice));
}

template <typename T>
void refresh_csrv(const DevCsrv<T> &d, const Csr &a, bool split_diag) {
  if (d.v == nullptr) return;
  std::vector<T> v, diag;
  if (split_diag) diag.assign(a.rows, T(0));
  for (int r = 0; r < a.rows; ++r)
    for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
      if (split_diag && a.ci[k] == r) {
        diag[r] = T(a.v[k]);
        continue;
      }
      v.push_back(T(a.v[k]));
    }
  if (!v.empty()) GSB_CK(cudaMemcpy(d.v, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  if (split_diag && d.diag != nullptr)
    GSB_CK(cudaMemcpy(d.diag, diag.data(), sizeof(T) * diag.size(), cudaMemcpyHostToDevice));
}

template <typename T>
void refresh_bell(const DevBell<T> &d, const Csr &a, const std::vector<int> &node_bounds) {
  if (d.val == nullptr) return;
  const HostBell<T> h = make_bell<T>(a, node_bounds, d.g);
  if (9LL * h.bptr.back() != d.stored) throw std::runtime_error("update_values: the matrix sparsity changed");
  GSB_CK(cudaMemcpy(d.val, h.val.data(), sizeof(T) * h.val.size(), cudaMemcpyHostToDevice));
  GSB_CK(cudaMemcpy(d.diag, h.diag.data(), sizeof(T) * h.diag.size(), cudaMemcpyHostToDevice));
  GSB_CK(cudaMemcpy(d.dinv, h.dinv.data(), sizeof(T) * h.dinv.size(), cudaMemcpyHostToDevice));
}

// Off-diagonal block values of the block CSR-vector copy (diag and dinv are
// the BELL copy's arrays, refreshed with it).
template <typename T>
void refresh_bsrv(const DevBsrv<T> &d, const Csr &a) {
  if (d.v == nullptr) return;
  const int nn = a.rows / 3;
  std::vector<T> v;
  std::vector<int> cols;
  for (int I = 0; I < nn; ++I) {
    cols.clear();
    for (int r = 3 * I; r < 3 * I + 3; ++r)
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k)
        if (a.ci[k] / 3 != I) cols.push_back(a.ci[k] / 3);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const size_t base = v.size();
    v.resize(base + 9 * cols.size(), T(0));
    for (int r = 0; r < 3; ++r)
      for (int k = a.rp[3 * I + r]; k < a.rp[3 * I + r + 1]; ++k) {
        const int J = a.ci[k] / 3;
        if (J == I) continue;
        const size_t q = std::lower_bound(cols.begin(), cols.end(), J) - cols.begin();
        v[base + 9 * q + 3 * r + a.ci[k] % 3] = T(a.v[k]);
      }
  }
  if (!v.empty()) GSB_CK(cudaMemcpy(d.v, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------------------
// the solver, templated on the V-cycle precision
// ---------------------------------------------------------------------------
template <typename VT>
class AmgPcg final : public Solver {
 public:
  AmgPcg(const Hierarchy &h, const std::vector<const int *> &o2n,
         const std::vector<const int *> &n2o, const SolverOptions &opt, int device);
  ~AmgPcg() override;

  void solve_device(const double *b, double *x, cudaStream_t stream, SolveStats *st) override;
  void solve_host(const double *b, double *x, SolveStats *st) override;
  void apply_preconditioner(const double *r, double *z, cudaStream_t stream) override;
  double time_kernel(int kind, int reps, cudaStream_t stream) override;
  double time_level(int level, int op, int lanes, int reps, cudaStream_t stream) override;
  std::vector<double> setup_times() const override { return setup_ms_; }
  // A^-1 of the SPD level matrix, computed in FP64 (host Cholesky up to
  // kHostInverseRows rows, else on the GPU) and stored as VT at `out`:
  // n * n row-major, or lower-triangle tiles when `packed`.
  void dense_inverse_into(const Csr &a, VT *out, bool packed, __half *out_h = nullptr, float *scales = nullptr);
  void set_weights(const ColourWeights &w) override;
  void update_values(const double *a0_values) override;
  std::vector<LevelInfo> level_info() const override { return info_; }
  int device() const override { return device_; }
  int rows() const override { return n0_; }
  const SolverOptions &options() const override { return opt_; }
  long long launches() const override { return launches_; }
  std::vector<float> colour_features() const override { return features_; }
  std::vector<float> node_features() const override { return node_features_; }
  void set_node_weights(const std::vector<double> &w) override;
  double error_reduction(const double *e0, cudaStream_t stream) override;
  void set_tolerance(double tol, int max_iter) override {
    opt_.tol = tol;
    opt_.max_iter = max_iter;
  }

 private:
  struct Level {
    int n = 0, ncolors = 0;
    std::vector<int> color_slice;  // ncolors + 1
    std::vector<int> color_first;  // ncolors + 1: first row (scalar) or node (block)
    DevSell<VT> A;     // sliced layout in use (A.g lanes per row), scalar levels
    DevBell<VT> B;     // sliced layout in use (B.g lanes per node), 3x3 levels
    DevSell<VT> A1;    // the one-lane-per-row copies (A / B when g == 1)
    DevBell<VT> B1;
    DevCsrv<VT> C;     // CSR-vector copy of A (scalar levels)
    DevBsrv<VT> Bv;    // block-CSR-vector copy of A (3x3 levels)
    int kind = 0;        // smoother: 0 SGS, 1 block SGS, 2 damped Jacobi, 3 block Jacobi, 4 identity
    VT *jdinv = nullptr; // 1 / a_ii (damped Jacobi levels)
    bool sliced = true;  // A / B (SELL / BELL) or C / Bv (CSR-vector) in the smoother and residual
    int g = 1;           // lanes per row (node): 1, 2, 4, 8 sliced; 4, 8, 16, 32 CSR-vector
    DevSell<VT> P, R;  // to the next level
    DevCsrv<VT> Pc, Rc;
    int pg = 1, rg = 1;
    VT *x = nullptr, *b = nullptr, *r = nullptr;
    VT *ainv = nullptr;  // dense inverse of the coarsest level, in the V-cycle's precision
    bool packed = false;           // ainv in lower-triangle tiles (n > kPackedDenseRows)
    double *dense_partial = nullptr;  // tiles^2 x kDenseTile partial sums of the packed solve
    float *dense_partial_f = nullptr; // the same in FP32, for the FP16 tiles' tensor-core apply
    uint4 *dense_frag = nullptr;      // the vector's MMA fragments, 256 bytes per 64-entry chunk
    float *dense_inv = nullptr;       // and the inverse scale of each chunk
    __half *ainv_h = nullptr;         // packed tiles in FP16 (coarse_half), with one scale per tile
    float *ainv_scale = nullptr;
    std::vector<VT *> wts;  // per colour: device pointer to the weight, or nullptr
    bool coop = false;      // symmetric sweeps as one cooperative launch (scalar SGS levels)
    // colouring of the strong couplings only (coloring 2): a pass reads its
    // own colour's neighbours from `xprev`, the iterate its sweep started with
    bool relaxed = false;
    VT *xprev = nullptr;
    bool staged = false;    // 3x3 block passes with the slice's blocks bulk-copied to shared memory (BELL-1)
    VT *nwts = nullptr;     // learned scaling per node (3x3 block levels), internal order, or nullptr
    VT *nwts_buf = nullptr; // its device buffer, kept once allocated
    int *d_color_slice = nullptr, *d_color_first = nullptr;  // ncolors + 1 each, on the device
  };

  // dir: 0 symmetric steps (forward then backward colours), 1 forward
  // sweeps only, 2 backward sweeps only (half_sweeps pre / post smoothing)
  template <typename BT>
  void smooth(Level &L, const BT *rhs, VT *x, int steps, bool zero, cudaStream_t s, int dir = 0);
  template <typename BT>
  void gs_pass(Level &L, int c, const BT *rhs, VT *x, bool zero, cudaStream_t s);
  template <typename BT>
  void coop_sweep(Level &L, const BT *rhs, VT *x, int steps, bool zero, bool forward_only, cudaStream_t s);
  // omega 1 and no learned weight: the update of a row does not depend on
  // its own value, so a colour pass repeated right after itself (where the
  // sweep turns) reproduces its input bit for bit and is skipped
  bool skip_repeats(const Level &L) const {
    return VT(opt_.omega) == VT(1) && (L.wts.empty() || L.wts[0] == nullptr) && L.nwts == nullptr && !L.relaxed;
  }
  // x as the next sweep starts, for the same-colour reads of a relaxed level
  void sweep_start(Level &L, const VT *x, cudaStream_t s) {
    if (L.relaxed) CK(cudaMemcpyAsync(L.xprev, x, sizeof(VT) * L.n, cudaMemcpyDeviceToDevice, s));
  }
  void forward_sweep(Level &L, cudaStream_t s);
  void check_sync_fault(const CgState &hs);
  void drop_graphs();
  template <typename BT>
  void dense_coarse(Level &L, const BT *rhs, VT *x, cudaStream_t s);
  template <typename BT>
  void vcycle(int k, const BT *rhs, VT *x, bool zero, cudaStream_t s);
  template <typename BT>
  void level_spmv_resid(Level &L, const BT *rhs, const VT *x, VT *r, cudaStream_t s);
  void precondition(const double *r, VT *z, cudaStream_t s);
  template <int kMode, typename BT>
  void transfer(const DevSell<VT> &S, const DevCsrv<VT> &Cm, int g, const VT *x, VT *y, const BT *b,
                cudaStream_t s);
  void autotune();
  float time_ms(const std::function<void()> &f, int reps);
  void cg_iteration(int parity, cudaStream_t s);
  void cg_start(cudaStream_t s);
  void ensure_graphs();
  void run(cudaStream_t user, SolveStats *st);

  SolverOptions opt_;
  int device_ = 0, sms_ = 148, cap_blocks_ = 148 * 8;
  int n0_ = 0;
  bool block_ = false;
  // V-cycle kernels launched with programmatic stream serialization. Only
  // outside stream capture: replayed from a CUDA graph the kernels already
  // follow each other closely, and programmatic edges measured no faster.
  // setup wall-clock ms: 0 levels, 1 autotune, 2 coarse tail, 3 total, and
  // inside the levels 4 colouring, 5 permutations, 6 smoother features,
  // 7 smoother / residual layouts, 8 transfer layouts, 9 dense coarsest inverse
  std::vector<double> setup_ms_ = std::vector<double>(10, 0.0);
  std::vector<std::unique_ptr<Arena>> kept_layouts_;  // autotuner winners built in trial arenas
  bool pdl_ = true;
  struct PlainLaunches {  // clears pdl_ for the duration of a capture unless `keep`
    bool &flag;
    const bool saved;
    PlainLaunches(bool &f, bool keep) : flag(f), saved(f) { flag = flag && keep; }
    ~PlainLaunches() { flag = saved; }
  };
  Arena ar_;
  std::vector<Level> lv_;
  std::vector<LevelInfo> info_;
  // outer CG, FP64, internal order
  DevSell<double> cgA_;
  DevBell<double> cgB_;   // 3x3 block operator of the outer CG, BELL-32 with cgB_.g lanes per node
  std::unique_ptr<Arena> cg_arena_;  // cgB_ when the autotuner chose more than one lane per node
  void outer_spmv(const double *v, CgState *st, cudaStream_t s);
  void set_outer_lanes(int g);
  void tune_outer();
  void outer_resid(cudaStream_t s);
  double *x_ = nullptr, *r_ = nullptr, *p_ = nullptr, *ap_ = nullptr, *b_ = nullptr;
  VT *z_[2] = {nullptr, nullptr};
  double *ubuf_ = nullptr, *uxbuf_ = nullptr;  // caller-order staging for host solves
  int *q0_ = nullptr;                           // internal index of caller row i
  CgState *st_ = nullptr, *scratch_st_ = nullptr;
  double *partials_ = nullptr;
  CgState *host_st_ = nullptr;                  // pinned, two slots
  SweepSync *sync_ = nullptr;                   // grid-barrier state of the cooperative sweeps
  VT *wbuf_ = nullptr;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraph_t graph_[2] = {nullptr, nullptr};
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
  // cluster-resident coarse tail
  int tail_k0_ = -1;             // first level of the tail, -1 = no tail
  int tail_cluster_ = 0;         // CTAs per cluster (16 or 8)
  size_t tail_smem_ = 0;         // dynamic shared memory of the tail launch (x replicas)
  bool tail_on_ = false;
  int tail_cluster_size(size_t smem, int want);
  float time_segment(const std::function<void()> &f, int reps, int trials = 1);
  void upload_tail_table(int k0);
  TailLevel<VT> *tail_lv_ = nullptr;
  void setup_tail();
  std::string signature() const;
  void set_color_slices(Level &L);
  void set_layout(Level &L, int k, bool sliced, int g, Arena &where);
  std::vector<Csr> host_A_;  // level matrices in internal order, until the layouts are chosen
  // kept for update_values: internal order of every level, the transfer
  // operators (caller order) and the finest level's sparsity
  std::vector<std::vector<int>> Q_;
  std::vector<Csr> hP_, hR_;
  Csr hA0_;
  void launch_tail(cudaStream_t s);
  std::vector<float> features_;  // 8 per (level, colour)
  std::vector<float> node_features_;  // 8 per node of every level (3x3 block hierarchies), caller order
  long long launches_ = 0;       // kernels issued (a graph replay adds its kernel count)
  long long graph_kernels_ = 0;  // kernels in one captured iteration
};

template <typename VT>
AmgPcg<VT>::AmgPcg(const Hierarchy &h, const std::vector<const int *> &o2n,
                   const std::vector<const int *> &n2o, const SolverOptions &opt, int device)
    : opt_(opt), device_(device) {
  using clock = std::chrono::steady_clock;
  const auto ms_since = [](clock::time_point t) {
    return std::chrono::duration<double, std::milli>(clock::now() - t).count();
  };
  const auto t_setup = clock::now();
  int L = static_cast<int>(h.A.size());
  if (L == 0) throw std::runtime_error("MultigridSmoother: empty hierarchy.");
  if (static_cast<int>(h.P.size()) + 1 != L || static_cast<int>(h.R.size()) + 1 != L)
    throw std::runtime_error("MultigridSmoother: invalid number of transfers.");
  if (static_cast<int>(o2n.size()) != L || static_cast<int>(n2o.size()) != L)
    throw std::runtime_error("MultigridSmoother: invalid number of permutations.");
  if (!(opt.omega > 0.0 && opt.omega < 2.0)) throw std::runtime_error("smoother: omega must be in (0, 2).");
  if (opt.pre < 1 || opt.post < 1 || opt.vcycles < 1 || (opt.coarse == 0 && opt.coarse_steps < 1))
    throw std::runtime_error("Preconditioner requires at least one smoothing step.");
  const int fine_kind = opt.smoother;
  const int coarse_kind = opt.coarse_smoother < 0 ? opt.smoother : opt.coarse_smoother;
  for (int kind : {fine_kind, coarse_kind})
    if (kind < 0 || kind > 4) throw std::runtime_error("MultigridSmoother: unsupported smoother type.");
  auto is_block = [](int kind) { return kind == 1 || kind == 3; };
  auto is_scalar = [](int kind) { return kind == 0 || kind == 2; };
  block_ = is_block(fine_kind) || (L > 1 && is_block(coarse_kind));
  if (block_ && (is_scalar(fine_kind) || (L > 1 && is_scalar(coarse_kind))))
    throw std::runtime_error("smoother: scalar and 3x3 block smoothers cannot be mixed in one hierarchy");
  if ((fine_kind == 4 || (L > 1 && coarse_kind == 4)) && L != 1)
    throw std::runtime_error("smoother: identity is a single-level preconditioner only");
  if (opt.coarse_rows < 0) throw std::runtime_error("coarse_rows must be >= 0");
  if (opt.coarse == 1) {
    std::vector<int> rows;
    for (const Csr &a : h.A) rows.push_back(a.rows);
    L = dense_depth(rows, opt.coarse_rows);
  }
  CK(cudaSetDevice(device_));
  sms_ = sm_count(device_);
  cap_blocks_ = sms_ * 8;
  if (opt.overlap_launch < 0 || opt.overlap_launch > 2) throw std::runtime_error("overlap_launch must be 0, 1 or 2");
  if (opt.packed_rows < 0) throw std::runtime_error("packed_rows must be >= 0");
  if (opt.coloring < 0 || opt.coloring > 2) throw std::runtime_error("coloring must be 0, 1 or 2");
  if (opt.sweep_launch < 0 || opt.sweep_launch > 2) throw std::runtime_error("sweep_launch must be 0, 1 or 2");
  if (opt.half_sweeps != 0 && opt.half_sweeps != 1) throw std::runtime_error("half_sweeps must be 0 or 1");
  if (opt.coarse_half != 0 && opt.coarse_half != 1) throw std::runtime_error("coarse_half must be 0 or 1");
  pdl_ = opt.overlap_launch >= 1;
  CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (auto &e : ev_) CK(cudaEventCreate(&e));
  lv_.resize(L);
  info_.resize(L);

  std::vector<std::vector<int>> Q(L);
  auto tick = clock::now();
  const auto lap = [&](int phase) {
    const auto now = clock::now();
    setup_ms_[phase] += std::chrono::duration<double, std::milli>(now - tick).count();
    tick = now;
  };
  for (int k = 0; k < L; ++k) {
    const Csr &Ak = h.A[k];
    Ak.check("hierarchy level matrix");
    if (Ak.rows != Ak.cols) throw std::runtime_error("level matrix must be square");
    const int n = Ak.rows;
    if (block_ && n % 3 != 0)
      throw std::runtime_error("BlockGaussSeidelSmoother: number of DOFs must be divisible by 3.");
    std::vector<int> id;
    const int *po = o2n[k], *pn = n2o[k];
    const bool identity = po == nullptr;
    if (identity) {
      id.resize(n);
      std::iota(id.begin(), id.end(), 0);
      po = pn = id.data();
    } else {
      check_permutation(n, po, pn);
    }
    // the colouring walks the permuted graph; without a permutation that is
    // the level itself (the order of columns within a row does not matter)
    Csr permuted;
    if (!identity) permuted = permute_matrix(Ak, po, po);
    const Csr &Ap = identity ? Ak : permuted;
    lap(5);
    std::vector<int> colors, verts, offs;
    int nc;
    {
      std::vector<int> grp, gci;
      if (block_) block_graph(Ap, 3, grp, gci);
      const int gn = block_ ? n / 3 : n;
      const int *grow = block_ ? grp.data() : Ap.rp.data();
      const int *gcol = block_ ? gci.data() : Ap.ci.data();
      const int kind_k = k == 0 ? fine_kind : coarse_kind;
      if (opt.coloring == 2 && k > 0 && kind_k == 0) {
        // coarse scalar Gauss-Seidel levels: colour the strong couplings only
        nc = relaxed_coloring(n, Ap.rp.data(), Ap.ci.data(), Ap.v.data(), kRelaxedTheta, kRelaxedRho, colors, verts,
                              offs);
        lv_[k].relaxed = true;
      } else if (opt.coloring == 2 && k > 0 && kind_k == 1) {
        // coarse block Gauss-Seidel levels: the nodes' strong block couplings
        nc = relaxed_block_coloring(Ap, kRelaxedTheta, kRelaxedRho, colors, verts, offs);
        lv_[k].relaxed = true;
      } else {
        nc = greedy_coloring(gn, grow, gcol, colors, verts, offs);
      }
      // coloring 1 (and 2 elsewhere): first-fit in smallest-last order where
      // it needs fewer colours; a level the greedy order already colours with
      // two (a bipartite graph: no colouring has fewer) skips the ordering
      if (opt.coloring >= 1 && !lv_[k].relaxed && nc > 2) {
        std::vector<int> c2, v2, o2;
        const int n2 = smallest_last_coloring(gn, grow, gcol, c2, v2, o2);
        if (n2 < nc) nc = n2, colors.swap(c2), verts.swap(v2), offs.swap(o2);
      }
    }
    lap(4);
    // gamma: position of each (node or row) of Ap in the colour-grouped list
    std::vector<int> gamma(verts.size());
    for (size_t i = 0; i < verts.size(); ++i) gamma[verts[i]] = static_cast<int>(i);
    Q[k].resize(n);
    for (int i = 0; i < n; ++i) {
      const int pi = po[i];
      Q[k][i] = block_ ? 3 * gamma[pi / 3] + pi % 3 : gamma[pi];
    }
    const Csr Ai = permute_matrix(Ak, Q[k].data(), Q[k].data());
    lap(5);
    append_colour_features(Ai, offs, block_ ? 3 : 1, k, L, features_);
    if (block_) append_node_features(Ai, offs, Q[k], k, L, node_features_);
    lap(6);
    Level &lv = lv_[k];
    lv.n = n;
    lv.ncolors = nc;
    lv.color_first = offs;
    lv.wts.assign(nc, nullptr);
    lv.kind = k == 0 ? fine_kind : coarse_kind;
    info_[k].rows = n;
    info_[k].nnz = Ai.nnz();
    info_[k].colors = nc;
    if (block_) {
      const HostBell<VT> hb = make_bell<VT>(Ai, offs);
      lv.B = upload_bell(ar_, hb);
      lv.Bv = upload_bsrv<VT>(ar_, Ai, lv.B);
      info_[k].slices = lv.B.nslices;
      info_[k].stored = lv.B.stored;
      if (k == 0) {
        cg_arena_.reset(new Arena);
        cgB_ = upload_bell(*cg_arena_, make_bell<double>(Ai, offs));
      }
    } else {
      for (int r = 0; r < n; ++r) {
        bool found = false;
        for (int e = Ai.rp[r]; e < Ai.rp[r + 1]; ++e)
          if (Ai.ci[e] == r && std::fabs(Ai.v[e]) >= 1e-12) found = true;
        if (!found) throw std::runtime_error("Gauss-Seidel: zero or missing diagonal entry.");
      }
      const HostSell<VT> hs = make_sell<VT>(Ai, offs, true);
      if (lv.kind == 2) {
        // DampedJacobiSmoother::initialize (src/Smoothers/DampedJacobiSmoother.cc:12-45)
        std::vector<VT> jd(n);
        for (int r = 0; r < n; ++r) jd[r] = VT(1) / hs.diag[r];
        lv.jdinv = ar_.upload(jd);
      }
      lv.A = upload_sell(ar_, hs);
      lv.C = upload_csrv<VT>(ar_, Ai, true);
      info_[k].slices = lv.A.nslices;
      info_[k].stored = lv.A.stored;
      if (k == 0) cgA_ = upload_sell(ar_, make_sell<double>(Ai, offs, true));
    }
    lv.A1 = lv.A;
    lv.B1 = lv.B;
    set_color_slices(lv);
    host_A_.push_back(Ai);  // kept until the layouts are chosen
    lv.x = ar_.alloc<VT>(n);
    lv.b = ar_.alloc<VT>(n);
    lv.r = ar_.alloc<VT>(n);
    if (lv.relaxed) {
      // defined before the first sweep fills it (the autotuner times passes
      // without the per-sweep copy)
      lv.xprev = ar_.alloc<VT>(n);
      CK(cudaMemset(lv.xprev, 0, sizeof(VT) * n));
    }
    lap(7);
    if (k > 0) {
      const Csr Pi = permute_matrix(h.P[k - 1], Q[k - 1].data(), Q[k].data());
      const Csr Ri = permute_matrix(h.R[k - 1], Q[k].data(), Q[k - 1].data());
      if (Pi.rows != lv_[k - 1].n || Pi.cols != n || Ri.rows != n || Ri.cols != lv_[k - 1].n)
        throw std::runtime_error("MultigridSmoother: transfer operator shape mismatch.");
      lv_[k - 1].P = upload_sell(ar_, make_sell<VT>(Pi, {0, Pi.rows}, false));
      lv_[k - 1].R = upload_sell(ar_, make_sell<VT>(Ri, {0, Ri.rows}, false));
      lv_[k - 1].Pc = upload_csrv<VT>(ar_, Pi, false);
      lv_[k - 1].Rc = upload_csrv<VT>(ar_, Ri, false);
    }
    lap(8);
    if (k == L - 1 && opt_.coarse == 1) {
      lv.packed = n > opt_.packed_rows;
      if (lv.packed) {
        const size_t tiles = (static_cast<size_t>(n) + kDenseTile - 1) / kDenseTile;
        const size_t elems = tiles * (tiles + 1) / 2 * kDenseTile * kDenseTile;
        if (opt_.coarse_half && sizeof(VT) == 4) {
          lv.ainv_h = ar_.alloc<__half>(elems);
          lv.ainv_scale = ar_.alloc<float>(tiles * (tiles + 1) / 2);
          lv.dense_partial_f = ar_.alloc<float>(tiles * tiles * kDenseTile);
          lv.dense_frag = ar_.alloc<uint4>(tiles * 16);
          lv.dense_inv = ar_.alloc<float>(tiles);
          CK(cudaFuncSetAttribute(dense_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dense_mma_smem())));
        } else {
          lv.ainv = ar_.alloc<VT>(elems);
          lv.dense_partial = ar_.alloc<double>(tiles * tiles * kDenseTile);
        }
      } else {
        lv.ainv = ar_.alloc<VT>(static_cast<size_t>(n) * n);
      }
      dense_inverse_into(Ai, lv.ainv, lv.packed, lv.ainv_h, lv.ainv_scale);
      CK(cudaDeviceSynchronize());
      lap(9);
    }
  }
  n0_ = lv_[0].n;
  x_ = ar_.alloc<double>(n0_);
  r_ = ar_.alloc<double>(n0_);
  p_ = ar_.alloc<double>(n0_);
  ap_ = ar_.alloc<double>(n0_);
  b_ = ar_.alloc<double>(n0_);
  z_[0] = ar_.alloc<VT>(n0_);
  z_[1] = ar_.alloc<VT>(n0_);
  ubuf_ = ar_.alloc<double>(n0_);
  uxbuf_ = ar_.alloc<double>(n0_);
  q0_ = ar_.upload(Q[0]);
  Q_ = Q;
  hA0_ = h.A[0];
  for (int k = 0; k + 1 < L; ++k) hP_.push_back(h.P[k]), hR_.push_back(h.R[k]);
  st_ = ar_.alloc<CgState>(1);
  scratch_st_ = ar_.alloc<CgState>(1);
  CK(cudaMemset(st_, 0, sizeof(CgState)));
  CK(cudaMemset(scratch_st_, 0, sizeof(CgState)));
  sync_ = ar_.alloc<SweepSync>(1);
  CK(cudaMemset(sync_, 0, sizeof(SweepSync)));
  partials_ = ar_.alloc<double>(3 * static_cast<size_t>(cap_blocks_) + 8);
  CK(cudaMallocHost(&host_st_, 2 * sizeof(CgState)));
  std::memset(host_st_, 0, 2 * sizeof(CgState));
  CK(cudaDeviceSynchronize());
  setup_ms_[0] = ms_since(t_setup);
  const auto t_tune = clock::now();
  if (opt_.sliced_lanes != 0 && opt_.sliced_lanes != 1 && opt_.sliced_lanes != 2 && opt_.sliced_lanes != 4 &&
      opt_.sliced_lanes != 8)
    throw std::runtime_error("sliced_lanes must be 0, 1, 2, 4 or 8");
  if (opt_.lanes > 0) {
    if (opt_.lanes != 1 && opt_.lanes != 4 && opt_.lanes != 8 && opt_.lanes != 16 && opt_.lanes != 32)
      throw std::runtime_error("lanes must be 1, 4, 8, 16 or 32");
    for (size_t k = 0; k < lv_.size(); ++k) {
      Level &l = lv_[k];
      l.pg = l.rg = opt_.lanes;
      set_layout(l, static_cast<int>(k), opt_.lanes == 1, opt_.lanes, ar_);
    }
  } else if (opt_.autotune) {
    autotune();
  }
  if (opt_.sliced_lanes > 0) {
    for (size_t k = 0; k < lv_.size(); ++k) set_layout(lv_[k], static_cast<int>(k), true, opt_.sliced_lanes, ar_);
    set_outer_lanes(opt_.sliced_lanes);
  }
  if (opt_.sweep_launch == 2)
    for (Level &l : lv_) {
      l.coop = l.kind == 0 && !block_ && !l.relaxed && !opt_.half_sweeps;
      l.staged = block_ && l.sliced && l.g == 1 && prepare_staged<VT>(l.B.max_slots, device_);
    }
  host_A_.clear();
  host_A_.shrink_to_fit();
  CK(cudaDeviceSynchronize());
  setup_ms_[1] = ms_since(t_tune);
  const auto t_tail = clock::now();
  bool all_sgs = true;
  for (const Level &l : lv_) all_sgs = all_sgs && l.kind == 0 && !l.relaxed;
  // the cluster-resident tail runs symmetric multicolour SGS steps only
  if (!block_ && all_sgs && !opt_.half_sweeps) setup_tail();
  CK(cudaDeviceSynchronize());
  setup_ms_[2] = ms_since(t_tail);
  setup_ms_[3] = ms_since(t_setup);
  for (size_t k = 0; k < lv_.size(); ++k) {
    info_[k].in_tail = tail_on_ && static_cast<int>(k) >= tail_k0_;
    info_[k].tail_ctas = info_[k].in_tail ? tail_cluster_ : 0;
    info_[k].lanes = lv_[k].g;
    info_[k].sliced = lv_[k].sliced ? 1 : 0;
    info_[k].launch = lv_[k].coop ? 1 : (lv_[k].staged ? 2 : 0);
    info_[k].p_lanes = lv_[k].pg;
    info_[k].r_lanes = lv_[k].rg;
  }
}

template <typename VT>
AmgPcg<VT>::~AmgPcg() {
  cudaSetDevice(device_);
  for (int i = 0; i < 2; ++i) {
    if (exec_[i]) cudaGraphExecDestroy(exec_[i]);
    if (graph_[i]) cudaGraphDestroy(graph_[i]);
  }
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  if (host_st_) cudaFreeHost(host_st_);
  if (stream_) cudaStreamDestroy(stream_);
}

template <typename VT>
void AmgPcg<VT>::dense_inverse_into(const Csr &a, VT *out, bool packed, __half *out_h, float *scales) {
  const size_t nn = static_cast<size_t>(a.rows) * a.rows;
  if (packed) {
    double *tmp = nullptr;
    CK(cudaMalloc(&tmp, sizeof(double) * nn));
    try {
      if (a.rows <= kHostInverseRows) {
        const std::vector<double> inv = cholesky_inverse(a);
        CK(cudaMemcpy(tmp, inv.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
      } else {
        spd_inverse_device(a, tmp, stream_, true);  // the packing reads the lower tiles only
      }
      const long long tiles = (a.rows + kDenseTile - 1) / kDenseTile;
      if (out_h != nullptr)
        dense_pack_kernel<__half><<<static_cast<unsigned>(tiles * (tiles + 1) / 2), 256, 0, stream_>>>(a.rows, tmp, out_h,
                                                                                                         scales);
      else
        dense_pack_kernel<VT><<<static_cast<unsigned>(tiles * (tiles + 1) / 2), 256, 0, stream_>>>(a.rows, tmp, out);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(stream_));
    } catch (...) {
      cudaFree(tmp);
      throw;
    }
    CK(cudaFree(tmp));
    return;
  }
  if (a.rows <= kHostInverseRows) {
    const std::vector<double> inv = cholesky_inverse(a);
    const std::vector<VT> cv(inv.begin(), inv.end());
    CK(cudaMemcpy(out, cv.data(), sizeof(VT) * nn, cudaMemcpyHostToDevice));
    return;
  }
  if (nn > 2147483647ull) throw std::runtime_error("dense coarsest level: more than 46340 rows");
  if (sizeof(VT) == sizeof(double)) {
    spd_inverse_device(a, reinterpret_cast<double *>(out), stream_);
    return;
  }
  double *tmp = nullptr;
  CK(cudaMalloc(&tmp, sizeof(double) * nn));
  try {
    spd_inverse_device(a, tmp, stream_);
    convert_kernel<VT, double><<<blocks_for(static_cast<long long>(nn), cap_blocks_), 256, 0, stream_>>>(
        static_cast<int>(nn), tmp, out, nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
  } catch (...) {
    cudaFree(tmp);
    throw;
  }
  CK(cudaFree(tmp));
}

template <typename VT>
void AmgPcg<VT>::update_values(const double *a0_values) {
  if (a0_values == nullptr) throw std::runtime_error("update_values: null values");
  CK(cudaSetDevice(device_));
  CK(cudaStreamSynchronize(stream_));
  const int L = static_cast<int>(lv_.size());
  Csr A0 = hA0_;
  std::memcpy(A0.v.data(), a0_values, sizeof(double) * A0.v.size());
  // the coarser levels R_k A_k P_k: the setup's sparse products on the GPU
  // (bit-identical to the host's); a product row of more than 1024 columns,
  // or unsorted caller rows, take the host's products instead
  std::vector<Csr> levels;
  try {
    levels = galerkin_device(A0, hP_, hR_, L, device_);
  } catch (const CudaError &) {
    throw;
  } catch (const std::runtime_error &) {
    levels.assign(1, A0);
    for (int k = 0; k + 1 < L; ++k) levels.push_back(spgemm(hR_[k], spgemm(levels[k], hP_[k])));
  }
  CK(cudaSetDevice(device_));
  std::vector<float> features, node_features;
  for (int k = 0; k < L; ++k) {
    Level &lv = lv_[k];
    const Csr &Ak = levels[k];
    const Csr Ai = permute_matrix(Ak, Q_[k].data(), Q_[k].data());
    if (block_) {
      refresh_bell(lv.B1, Ai, lv.color_first);
      if (lv.B.val != lv.B1.val) refresh_bell(lv.B, Ai, lv.color_first);
      refresh_bsrv(lv.Bv, Ai);
      if (k == 0) refresh_bell(cgB_, Ai, lv.color_first);
    } else {
      for (int r = 0; r < Ai.rows; ++r) {
        bool found = false;
        for (int e = Ai.rp[r]; e < Ai.rp[r + 1]; ++e)
          if (Ai.ci[e] == r && std::fabs(Ai.v[e]) >= 1e-12) found = true;
        if (!found) throw std::runtime_error("Gauss-Seidel: zero or missing diagonal entry.");
      }
      refresh_sell(lv.A1, Ai, lv.color_first, true);
      if (lv.A.val != lv.A1.val) refresh_sell(lv.A, Ai, lv.color_first, true);
      refresh_csrv(lv.C, Ai, true);
      if (k == 0) refresh_sell(cgA_, Ai, lv.color_first, true);
      if (lv.kind == 2) {
        std::vector<VT> jd(Ai.rows, VT(0));
        for (int r = 0; r < Ai.rows; ++r)
          for (int e = Ai.rp[r]; e < Ai.rp[r + 1]; ++e)
            if (Ai.ci[e] == r) jd[r] = VT(1) / VT(Ai.v[e]);
        CK(cudaMemcpy(lv.jdinv, jd.data(), sizeof(VT) * jd.size(), cudaMemcpyHostToDevice));
      }
    }
    append_colour_features(Ai, lv.color_first, block_ ? 3 : 1, k, L, features);
    if (block_) append_node_features(Ai, lv.color_first, Q_[k], k, L, node_features);
    if (k == L - 1 && opt_.coarse == 1) dense_inverse_into(Ai, lv.ainv, lv.packed, lv.ainv_h, lv.ainv_scale);
  }
  features_ = features;
  node_features_ = node_features;
}

template <typename VT>
void AmgPcg<VT>::set_weights(const ColourWeights &w) {
  if (w.w.empty()) {
    for (auto &l : lv_) std::fill(l.wts.begin(), l.wts.end(), nullptr);
    if (tail_on_) upload_tail_table(tail_k0_);
    drop_graphs();  // the captured kernels carry the weight pointers
    return;
  }
  const int L = static_cast<int>(lv_.size());
  if (static_cast<int>(w.level_offset.size()) != L + 1)
    throw std::runtime_error("colour weights: level offsets do not match the hierarchy");
  std::vector<VT> hv(w.w.size());
  for (size_t i = 0; i < w.w.size(); ++i) {
    if (!(w.w[i] > 0.0 && w.w[i] < 2.0)) throw std::runtime_error("colour weights must lie in (0, 2)");
    hv[i] = VT(w.w[i]);
  }
  for (int k = 0; k < L; ++k)
    if (w.level_offset[k + 1] - w.level_offset[k] != lv_[k].ncolors)
      throw std::runtime_error("colour weights: colour count mismatch");
  if (wbuf_ == nullptr) {
    size_t total = 0;
    for (auto &l : lv_) total += l.ncolors;
    wbuf_ = ar_.alloc<VT>(total);
  }
  CK(cudaMemcpy(wbuf_, hv.data(), hv.size() * sizeof(VT), cudaMemcpyHostToDevice));
  for (int k = 0; k < L; ++k)
    for (int c = 0; c < lv_[k].ncolors; ++c) lv_[k].wts[c] = wbuf_ + w.level_offset[k] + c;
  if (tail_on_) upload_tail_table(tail_k0_);  // the table carries the weight pointers
  drop_graphs();  // graphs bake the pointers in: rebuild on next use
}

// Learned scaling per node of the 3x3 block smoother, every level's nodes in
// the caller's order (the order of node_features); empty restores the colour
// weights / omega. Each level's weights go to the device in internal order.
template <typename VT>
void AmgPcg<VT>::set_node_weights(const std::vector<double> &w) {
  CK(cudaSetDevice(device_));
  if (w.empty()) {
    for (Level &l : lv_) l.nwts = nullptr;
    drop_graphs();
    return;
  }
  if (!block_) throw std::runtime_error("node weights: the hierarchy has no 3x3 block levels");
  size_t total = 0;
  for (const Level &l : lv_) total += static_cast<size_t>(l.n / 3);
  if (w.size() != total)
    throw std::runtime_error("node weights: expected " + std::to_string(total) + " values (one per node of every level)");
  for (double v : w)
    if (!(v > 0.0 && v < 2.0)) throw std::runtime_error("node weights must lie in (0, 2)");
  size_t base = 0;
  for (size_t k = 0; k < lv_.size(); ++k) {
    Level &l = lv_[k];
    const int nn = l.n / 3;
    std::vector<VT> hv(nn);
    for (int i = 0; i < nn; ++i) hv[Q_[k][3 * i] / 3] = VT(w[base + i]);
    if (l.nwts_buf == nullptr) l.nwts_buf = ar_.alloc<VT>(nn);
    CK(cudaMemcpy(l.nwts_buf, hv.data(), sizeof(VT) * nn, cudaMemcpyHostToDevice));
    l.nwts = l.nwts_buf;
    base += nn;
  }
  drop_graphs();
}

template <typename VT>
void AmgPcg<VT>::drop_graphs() {
  for (int i = 0; i < 2; ++i) {
    if (exec_[i]) cudaGraphExecDestroy(exec_[i]), exec_[i] = nullptr;
    if (graph_[i]) cudaGraphDestroy(graph_[i]), graph_[i] = nullptr;
  }
}

// Blocks of 256 threads of `kernel` resident on the whole GPU at once,
// queried from the runtime once per kernel: grid-stride kernels launched with
// at most this many blocks run as a single wave.
template <typename K>
int resident_grid(K kernel, int sms) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const void *key = reinterpret_cast<const void *>(kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0));
  const int g = std::max(1, per_sm) * sms;
  cache.emplace(key, g);
  return g;
}

template <typename VT>
template <typename BT>
void AmgPcg<VT>::gs_pass(Level &L, int c, const BT *rhs, VT *x, bool zero, cudaStream_t s) {
  const int s0 = L.color_slice[c], s1 = L.color_slice[c + 1];
  if (s1 <= s0) return;
  const VT *w = L.wts[c];
  const VT *nw = L.nwts;
  const VT *xp = L.relaxed ? L.xprev : nullptr;
  const VT om = VT(opt_.omega);
  const int *done = &st_->done;
  if (block_ && L.sliced && L.staged && L.g == 1) {
    const int ms = std::max(1, L.B.max_slots);
    const size_t smem = kStagedWarps * staged_warp_bytes<VT>(ms);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>((s1 - s0 + kStagedWarps - 1) / kStagedWarps));
    cfg.blockDim = dim3(32 * kStagedWarps);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = pdl_ ? attr : nullptr;
    cfg.numAttrs = pdl_ ? 1 : 0;
    if (zero)
      CK(cudaLaunchKernelEx(&cfg, bell_gs_staged_kernel<VT, BT, true>, L.B.view(), s0, s1, L.color_first[c], rhs, x, w,
                            om, st_, nw, ms, xp, L.color_first[c + 1]));
    else if (xp != nullptr)
      CK(cudaLaunchKernelEx(&cfg, bell_gs_staged_kernel<VT, BT, false, true>, L.B.view(), s0, s1, L.color_first[c], rhs,
                            x, w, om, st_, nw, ms, xp, L.color_first[c + 1]));
    else
      CK(cudaLaunchKernelEx(&cfg, bell_gs_staged_kernel<VT, BT, false>, L.B.view(), s0, s1, L.color_first[c], rhs, x,
                            w, om, st_, nw, ms, xp, L.color_first[c + 1]));
  } else if (block_ && L.sliced) {
    const int blocks = (s1 - s0 + 7) / 8;  // one warp per slice
#define GS_BELL(G)                                                                                              \
  if (zero) launch_pass(pdl_, bell_gs_kernel<VT, BT, true, G>, blocks, s, L.B.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, nw, xp, L.color_first[c + 1]); \
  else if (xp) launch_pass(pdl_, bell_gs_kernel<VT, BT, false, G, true>, blocks, s, L.B.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, nw, xp, L.color_first[c + 1]); \
  else launch_pass(pdl_, bell_gs_kernel<VT, BT, false, G>, blocks, s, L.B.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, nw, xp, L.color_first[c + 1]);
    switch (L.g) {
      case 1: GS_BELL(1) break;
      case 2: GS_BELL(2) break;
      case 4: GS_BELL(4) break;
      default: GS_BELL(8) break;
    }
#undef GS_BELL
  } else if (block_) {
    const int n0 = L.color_first[c], n1 = L.color_first[c + 1];
    const int gb = static_cast<int>((static_cast<long long>(n1 - n0) * L.g + 255) / 256);
    const BsrvView<VT> v = L.Bv.view();
#define GS_BSRV(G)                                                                                   \
  if (zero) launch_pass(pdl_, bsrv_gs_kernel<VT, BT, true, G>, gb, s, v, n0, n1, rhs, x, w, om, done, nw, xp);     \
  else if (xp) launch_pass(pdl_, bsrv_gs_kernel<VT, BT, false, G, true>, gb, s, v, n0, n1, rhs, x, w, om, done, nw, xp); \
  else launch_pass(pdl_, bsrv_gs_kernel<VT, BT, false, G>, gb, s, v, n0, n1, rhs, x, w, om, done, nw, xp);
    switch (L.g) {
      case 4: GS_BSRV(4) break;
      case 8: GS_BSRV(8) break;
      case 16: GS_BSRV(16) break;
      default: GS_BSRV(32) break;
    }
#undef GS_BSRV
  } else if (L.sliced) {
    // grid-stride over slices with at most one resident wave
#define GS_SELL(G)                                                                                        \
  {                                                                                                       \
    const int blocks = std::min((s1 - s0 + 7) / 8, sizeof(VT) == 4 ? cap_blocks_                          \
                                                   : resident_grid(sell_gs_kernel<VT, BT, false, G>, sms_)); \
    if (zero) launch_pass(pdl_, sell_gs_kernel<VT, BT, true, G>, blocks, s, L.A.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, xp, L.color_first[c + 1]); \
    else if (xp) launch_pass(pdl_, sell_gs_kernel<VT, BT, false, G, true>, blocks, s, L.A.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, xp, L.color_first[c + 1]); \
    else launch_pass(pdl_, sell_gs_kernel<VT, BT, false, G>, blocks, s, L.A.view(), s0, s1, L.color_first[c], rhs, x, w, om, done, xp, L.color_first[c + 1]); \
  }
    switch (L.g) {
      case 1: GS_SELL(1) break;
      case 2: GS_SELL(2) break;
      case 4: GS_SELL(4) break;
      default: GS_SELL(8) break;
    }
#undef GS_SELL
  } else {
    const int r0 = L.color_first[c], r1 = L.color_first[c + 1];
    const int gb = static_cast<int>((static_cast<long long>(r1 - r0) * L.g + 255) / 256);
    const CsrvView<VT> v = L.C.view();
#define GS_CSRV(G)                                                                                   \
  if (zero) launch_pass(pdl_, csrv_gs_kernel<VT, BT, true, G>, gb, s, v, r0, r1, rhs, x, w, om, done, xp);     \
  else if (xp) launch_pass(pdl_, csrv_gs_kernel<VT, BT, false, G, true>, gb, s, v, r0, r1, rhs, x, w, om, done, xp); \
  else launch_pass(pdl_, csrv_gs_kernel<VT, BT, false, G>, gb, s, v, r0, r1, rhs, x, w, om, done, xp);
    switch (L.g) {
      case 4: GS_CSRV(4) break;
      case 8: GS_CSRV(8) break;
      case 16: GS_CSRV(16) break;
      default: GS_CSRV(32) break;
    }
#undef GS_CSRV
  }
  CKL("gauss-seidel colour pass");
}

// SymmetricGaussSeidelSmoother::smooth / BlockGaussSeidelSmoother::smooth:
// each step is a forward sweep over colours 0..C-1 then a backward sweep.
template <typename VT>
template <typename BT>
void AmgPcg<VT>::smooth(Level &L, const BT *rhs, VT *x, int steps, bool zero, cudaStream_t s, int dir) {
  const int *done = &st_->done;
  if (L.kind == 4) {  // IdentityPreconditioner::apply
    launch_pass(pdl_, convert_kernel<VT, BT>, blocks_for(L.n, cap_blocks_), s, L.n, rhs, x, done);
    CKL("identity");
    return;
  }
  if (L.kind == 2 || L.kind == 3) {
    // DampedJacobiSmoother::smooth / BlockJacobiSmoother::smooth: per step
    // r = b - A x (the level's residual kernel), x += w D^-1 r; from a zero x
    // the first step is x = w D^-1 b
    const VT w = VT(opt_.omega);
    const VT *dinv = L.kind == 2 ? L.jdinv : (L.sliced ? L.B.dinv : L.Bv.dinv);
    const int units = L.kind == 2 ? L.n : L.n / 3;
    const int gb = blocks_for(units, cap_blocks_);
    for (int step = 0; step < steps; ++step) {
      if (zero && step == 0) {
        if (L.kind == 2) launch_pass(pdl_, jacobi_kernel<VT, BT, true>, gb, s, units, dinv, rhs, x, w, done);
        else launch_pass(pdl_, block_jacobi_kernel<VT, BT, true>, gb, s, units, dinv, rhs, x, w, done);
      } else {
        level_spmv_resid<BT>(L, rhs, x, L.r, s);
        if (L.kind == 2) launch_pass(pdl_, jacobi_kernel<VT, VT, false>, gb, s, units, dinv, L.r, x, w, done);
        else launch_pass(pdl_, block_jacobi_kernel<VT, VT, false>, gb, s, units, dinv, L.r, x, w, done);
      }
      CKL("jacobi step");
    }
    return;
  }
  if (dir != 0) {
    if (zero && dir == 2) throw std::runtime_error("smoother: a backward sweep from a zero iterate is not supported");
    // one direction per step: consecutive passes never repeat a colour
    for (int step = 0; step < steps; ++step) {
      const bool zs = zero && step == 0 && dir == 1;
      if (!zs) sweep_start(L, x, s);  // from zero the own colour is skipped anyway
      for (int i = 0; i < L.ncolors; ++i) {
        const int c = dir == 1 ? i : L.ncolors - 1 - i;
        // from a zero iterate the first forward sweep skips the later colours'
        // gathers; a backward sweep from zero has no such shortcut
        gs_pass(L, c, rhs, x, zs, s);
      }
    }
    return;
  }
  if (L.coop && L.kind == 0 && !block_ && !L.relaxed) {
    coop_sweep(L, rhs, x, steps, zero, false, s);
    return;
  }
  const bool skip = skip_repeats(L);
  for (int step = 0; step < steps; ++step) {
    if (!(zero && step == 0)) sweep_start(L, x, s);
    for (int c = 0; c < L.ncolors; ++c) {
      if (skip && step > 0 && c == 0) continue;  // the backward sweep just ended with colour 0
      gs_pass(L, c, rhs, x, zero && step == 0, s);
    }
    sweep_start(L, x, s);
    for (int c = L.ncolors - 1; c >= 0; --c) {
      if (skip && c == L.ncolors - 1) continue;  // the forward sweep just ended with this colour
      gs_pass(L, c, rhs, x, false, s);
    }
  }
}

// Co-resident blocks of kSweepThreads threads of `kernel` on the whole GPU.
template <typename K>
int coop_capacity(K kernel, int sms) {
  static std::mutex mu;
  static std::unordered_map<const void *, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const void *key = reinterpret_cast<const void *>(kernel);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSweepThreads, 0));
  const int g = per_sm * sms;
  cache.emplace(key, g);
  return g;
}

template <typename K, typename... A>
void launch_coop(K kernel, int grid, cudaStream_t s, A &&...args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(grid));
  cfg.blockDim = dim3(kSweepThreads);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

// `steps` symmetric Gauss-Seidel steps of a scalar level (or one forward
// sweep) in one cooperative launch (sweep.cuh); the same iterate as the
// per-colour passes, bit for bit.
template <typename VT>
template <typename BT>
void AmgPcg<VT>::coop_sweep(Level &L, const BT *rhs, VT *x, int steps, bool zero, bool forward_only,
                            cudaStream_t s) {
  SweepPlan plan;
  plan.bounds = L.sliced ? L.d_color_slice : L.d_color_first;
  plan.first_row = L.d_color_first;
  plan.ncolors = L.ncolors;
  plan.steps = steps;
  plan.zero = zero ? 1 : 0;
  plan.skip = skip_repeats(L) ? 1 : 0;
  plan.forward_only = forward_only ? 1 : 0;
  const VT *w = L.wts.empty() ? nullptr : L.wts[0];
  const VT om = VT(opt_.omega);
  // the whole co-resident grid: every colour is spread over all SMs
  auto go = [&](auto kernel, auto view) {
    const int grid = coop_capacity(kernel, sms_);
    if (grid < 1) throw std::runtime_error("cooperative sweep: kernel does not fit on an SM");
    launch_coop(kernel, grid, s, view, plan, rhs, x, w, om, st_, sync_);
  };
  if (L.sliced) {
    switch (L.g) {
      case 1: go(sell_sweep_kernel<VT, BT, 1>, L.A.view()); break;
      case 2: go(sell_sweep_kernel<VT, BT, 2>, L.A.view()); break;
      case 4: go(sell_sweep_kernel<VT, BT, 4>, L.A.view()); break;
      default: go(sell_sweep_kernel<VT, BT, 8>, L.A.view()); break;
    }
  } else {
    switch (L.g) {
      case 4: go(csrv_sweep_kernel<VT, BT, 4>, L.C.view()); break;
      case 8: go(csrv_sweep_kernel<VT, BT, 8>, L.C.view()); break;
      case 16: go(csrv_sweep_kernel<VT, BT, 16>, L.C.view()); break;
      default: go(csrv_sweep_kernel<VT, BT, 32>, L.C.view()); break;
    }
  }
  CKL("cooperative Gauss-Seidel sweep");
}

// One forward sweep over all colours of a level (the timing helpers).
template <typename VT>
void AmgPcg<VT>::forward_sweep(Level &L, cudaStream_t s) {
  if (L.coop && L.kind == 0 && !block_ && !L.relaxed) {
    coop_sweep<VT>(L, L.b, L.x, 1, false, true, s);
    return;
  }
  for (int c = 0; c < L.ncolors; ++c) gs_pass<VT>(L, c, L.b, L.x, false, s);
}

// A grid-barrier wait that gave up leaves the barrier state undefined: it is
// cleared before the error is reported, so the solver stays usable.
template <typename VT>
void AmgPcg<VT>::check_sync_fault(const CgState &hs) {
  if (hs.sync_fault == 0) return;
  CK(cudaStreamSynchronize(stream_));
  CK(cudaMemset(sync_, 0, sizeof(SweepSync)));
  CK(cudaMemset(st_, 0, sizeof(CgState)));
  throw CudaError("cooperative Gauss-Seidel sweep: a grid-barrier wait timed out");
}

template <typename VT>
template <typename BT>
void AmgPcg<VT>::level_spmv_resid(Level &L, const BT *rhs, const VT *x, VT *r, cudaStream_t s) {
  const int *done = &st_->done;
  if (block_ && L.sliced) {
    const int gb = blocks_for(32LL * L.B.nslices, cap_blocks_);
    switch (L.g) {
      case 1: launch_pass(pdl_, bell_spmv_kernel<VT, BT, kSpmvResid, 1>, gb, s, L.B.view(), x, r, rhs, done); break;
      case 2: launch_pass(pdl_, bell_spmv_kernel<VT, BT, kSpmvResid, 2>, gb, s, L.B.view(), x, r, rhs, done); break;
      case 4: launch_pass(pdl_, bell_spmv_kernel<VT, BT, kSpmvResid, 4>, gb, s, L.B.view(), x, r, rhs, done); break;
      default: launch_pass(pdl_, bell_spmv_kernel<VT, BT, kSpmvResid, 8>, gb, s, L.B.view(), x, r, rhs, done); break;
    }
  } else if (block_) {
    const int gb = blocks_for(static_cast<long long>(L.Bv.nodes) * L.g, cap_blocks_);
    switch (L.g) {
      case 4: launch_pass(pdl_, bsrv_spmv_kernel<VT, BT, kSpmvResid, 4>, gb, s, L.Bv.view(), x, r, rhs, done); break;
      case 8: launch_pass(pdl_, bsrv_spmv_kernel<VT, BT, kSpmvResid, 8>, gb, s, L.Bv.view(), x, r, rhs, done); break;
      case 16: launch_pass(pdl_, bsrv_spmv_kernel<VT, BT, kSpmvResid, 16>, gb, s, L.Bv.view(), x, r, rhs, done); break;
      default: launch_pass(pdl_, bsrv_spmv_kernel<VT, BT, kSpmvResid, 32>, gb, s, L.Bv.view(), x, r, rhs, done); break;
    }
  } else if (L.sliced) {
    const int gb = blocks_for(32LL * L.A.nslices, cap_blocks_);
    switch (L.g) {
      case 1: launch_pass(pdl_, sell_spmv_kernel<VT, BT, kSpmvResid, 1>, gb, s, L.A.view(), x, r, rhs, done); break;
      case 2: launch_pass(pdl_, sell_spmv_kernel<VT, BT, kSpmvResid, 2>, gb, s, L.A.view(), x, r, rhs, done); break;
      case 4: launch_pass(pdl_, sell_spmv_kernel<VT, BT, kSpmvResid, 4>, gb, s, L.A.view(), x, r, rhs, done); break;
      default: launch_pass(pdl_, sell_spmv_kernel<VT, BT, kSpmvResid, 8>, gb, s, L.A.view(), x, r, rhs, done); break;
    }
  } else {
    transfer<kSpmvResid, BT>(L.A1, L.C, L.g, x, r, rhs, s);
  }
  CKL("residual");
}

// x = A^-1 rhs on the dense coarsest level: full row-major inverse, or the
// packed lower-triangle tiles and their per-row reduction.
template <typename VT>
template <typename BT>
void AmgPcg<VT>::dense_coarse(Level &L, const BT *rhs, VT *x, cudaStream_t s) {
  const int *done = &st_->done;
  if (L.packed) {
    const int tiles = (L.n + kDenseTile - 1) / kDenseTile;
    const long long total = static_cast<long long>(tiles) * (tiles + 1) / 2;
    if (L.ainv_h != nullptr) {
      // FP16 tiles on the tensor cores: persistent warps, two CTAs per SM
      const long long ctas = std::min<long long>(2LL * sms_, (total + kMmaWarps - 1) / kMmaWarps);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(static_cast<unsigned>(ctas));
      cfg.blockDim = dim3(32 * kMmaWarps);
      cfg.dynamicSmemBytes = dense_mma_smem();
      cfg.stream = s;
      cfg.attrs = pdl_ ? attr : nullptr;
      cfg.numAttrs = pdl_ ? 1 : 0;
      launch_pass(pdl_, dense_vec_kernel<BT>, (tiles + 7) / 8, s, L.n, tiles, rhs, L.dense_frag, L.dense_inv, done);
      CKL("coarse solve (vector fragments)");
      CK(cudaLaunchKernelEx(&cfg, dense_mma_kernel, tiles, static_cast<const __half *>(L.ainv_h),
                            static_cast<const float *>(L.ainv_scale), static_cast<const uint4 *>(L.dense_frag),
                            static_cast<const float *>(L.dense_inv), L.dense_partial_f, st_));
      CKL("coarse solve (tensor-core tiles)");
      launch_pass(pdl_, dense_reduce_kernel<VT, float>, tiles, s, L.n, tiles, static_cast<const float *>(L.dense_partial_f),
                  x, done);
    } else {
      constexpr int kT = dense_tiles_per_cta<VT>();
      launch_pass(pdl_, dense_tile_kernel<BT, VT, VT>, static_cast<int>((total + kT - 1) / kT), s, L.n, tiles, L.ainv,
                  rhs, L.dense_partial, done, static_cast<const float *>(nullptr));
      CKL("coarse solve (tiles)");
      launch_pass(pdl_, dense_reduce_kernel<VT>, tiles, s, L.n, tiles, static_cast<const double *>(L.dense_partial), x,
                  done);
    }
    CKL("coarse solve (reduce)");
  } else {
    launch_pass(pdl_, dense_solve_kernel<BT, VT>, (L.n + 7) / 8, s, L.n, L.ainv, rhs, x, done);
    CKL("coarse solve");
  }
}

// MultigridSmoother::vCycle (src/Smoothers/MultigridSmoother.cc:337-412).
// `zero`: x is an implicit zero vector on entry (the preconditioner zeroes z,
// and every coarse correction starts from zero).
template <typename VT>
template <typename BT>
void AmgPcg<VT>::vcycle(int k, const BT *rhs, VT *x, bool zero, cudaStream_t s) {
  Level &L = lv_[k];
  if (tail_on_ && k == tail_k0_) {
    launch_tail(s);  // the whole V-cycle of levels k..L-1, x_k from a zero guess
    return;
  }
  const bool coarsest = k + 1 == static_cast<int>(lv_.size());
  if (coarsest) {
    if (opt_.coarse == 1) {
      dense_coarse<BT>(L, rhs, x, s);
    } else {
      smooth(L, rhs, x, opt_.coarse_steps, zero, s);
    }
    return;
  }
  smooth(L, rhs, x, opt_.pre, zero, s, opt_.half_sweeps ? 1 : 0);
  level_spmv_resid(L, rhs, x, L.r, s);
  Level &C = lv_[k + 1];
  transfer<kSpmvSet, VT>(L.R, L.Rc, L.rg, L.r, C.b, (const VT *)nullptr, s);
  CKL("restriction");
  vcycle<VT>(k + 1, C.b, C.x, true, s);
  if (opt_.reference_vcycle && k > 0)
    transfer<kSpmvTwice, VT>(L.P, L.Pc, L.pg, C.x, x, (const VT *)nullptr, s);
  else
    transfer<kSpmvAdd, VT>(L.P, L.Pc, L.pg, C.x, x, (const VT *)nullptr, s);
  CKL("prolongation");
  smooth(L, rhs, x, opt_.post, false, s, opt_.half_sweeps ? 2 : 0);
}

// y (op)= M x with M in SELL-32 (g == 1) or CSR-vector with g lanes per row.
template <typename VT>
template <int kMode, typename BT>
void AmgPcg<VT>::transfer(const DevSell<VT> &S, const DevCsrv<VT> &Cm, int g, const VT *x, VT *y,
                          const BT *b, cudaStream_t s) {
  const int *done = &st_->done;
  if (g == 1) {
    launch_pass(pdl_, sell_spmv_kernel<VT, BT, kMode>, blocks_for(32LL * S.nslices, cap_blocks_), s, S.view(), x, y, b, done);
    return;
  }
  const int gb = blocks_for(static_cast<long long>(Cm.rows) * g, cap_blocks_);
  switch (g) {
    case 4: launch_pass(pdl_, csrv_spmv_kernel<VT, BT, kMode, 4>, gb, s, Cm.view(), x, y, b, done); break;
    case 8: launch_pass(pdl_, csrv_spmv_kernel<VT, BT, kMode, 8>, gb, s, Cm.view(), x, y, b, done); break;
    case 16: launch_pass(pdl_, csrv_spmv_kernel<VT, BT, kMode, 16>, gb, s, Cm.view(), x, y, b, done); break;
    default: launch_pass(pdl_, csrv_spmv_kernel<VT, BT, kMode, 32>, gb, s, Cm.view(), x, y, b, done); break;
  }
}

template <typename VT>
float AmgPcg<VT>::time_ms(const std::function<void()> &f, int reps) {
  f();
  CK(cudaEventRecord(ev_[2], stream_));
  for (int i = 0; i < reps; ++i) f();
  CK(cudaEventRecord(ev_[3], stream_));
  CK(cudaEventSynchronize(ev_[3]));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
  return ms / reps;
}

// Threads per row, per level and per transfer operator: every candidate
// (SELL-32 with one lane per row, CSR-vector with 4/8/16/32 lanes) runs a
// full forward Gauss-Seidel sweep (or one SpMV for P and R) on the solver's
// own buffers, timed with CUDA events; the fastest wins. The sweep results
// are discarded (the level vectors are scratch until the first solve).
// Signature of this hierarchy for the decision cache: precision, levels and
// each level's rows, nonzeros and colours.
template <typename VT>
std::string AmgPcg<VT>::signature() const {
  std::ostringstream sig;
  sig << (sizeof(VT) == 4 ? "f32" : "f64") << ":" << lv_.size();
  for (size_t k = 0; k < lv_.size(); ++k)
    sig << ":" << lv_[k].n << "/" << info_[k].nnz << "/" << lv_[k].ncolors;
  return sig.str();
}

// Colour -> slice range of the sliced layout in use.
template <typename VT>
void AmgPcg<VT>::set_color_slices(Level &L) {
  const std::vector<int> &srow = block_ ? L.B.h_srow : L.A.h_srow;
  L.color_slice.resize(L.ncolors + 1);
  for (int c = 0; c <= L.ncolors; ++c)
    L.color_slice[c] =
        static_cast<int>(std::lower_bound(srow.begin(), srow.end(), L.color_first[c]) - srow.begin());
  // the cooperative sweep reads the colour bounds on the device
  if (L.d_color_slice == nullptr) {
    L.d_color_slice = ar_.alloc<int>(L.ncolors + 1);
    L.d_color_first = ar_.alloc<int>(L.ncolors + 1);
  }
  CK(cudaMemcpy(L.d_color_slice, L.color_slice.data(), sizeof(int) * (L.ncolors + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(L.d_color_first, L.color_first.data(), sizeof(int) * (L.ncolors + 1), cudaMemcpyHostToDevice));
}

// Smoother / residual layout of level k: sliced (SELL / BELL with g lanes per
// row or node, built from the level's host matrix into `where` when g > 1)
// or CSR-vector with g lanes.
template <typename VT>
void AmgPcg<VT>::set_layout(Level &L, int k, bool sliced, int g, Arena &where) {
  L.sliced = sliced;
  L.g = g;
  if (!sliced) return;
  if (g == 1) {
    L.A = L.A1;
    L.B = L.B1;
  } else if (block_) {
    if (L.B.g != g) L.B = upload_bell(where, make_bell<VT>(host_A_.at(k), L.color_first, g));
  } else {
    if (L.A.g != g) L.A = upload_sell(where, make_sell<VT>(host_A_.at(k), L.color_first, true, g));
  }
  set_color_slices(L);
}

// Format of every level's smoother and residual and of every transfer
// operator: each candidate -- sliced (SELL-32 / BELL-32 with 1, 2, 4 or 8
// lanes per row or node) and CSR-vector with 4, 8, 16 or 32 lanes -- runs a
// full forward Gauss-Seidel sweep (one SpMV for P and R) on the solver's own
// buffers, 10 times, launched as the solve launches it (replayed from a
// captured graph in graph mode), timed with CUDA events; the fastest wins.
template <typename VT>
void AmgPcg<VT>::autotune() {
  static const int cands[] = {1, 4, 8, 16, 32};
  const std::string sig = "v4:" + signature();
  if (!opt_.tune_cache.empty()) {
    std::ifstream in(opt_.tune_cache);
    std::string key, line;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      ls >> key;
      if (key != sig) continue;
      std::vector<int> v(6 * lv_.size() + 1);
      for (int &t : v) ls >> t;
      if (!ls) continue;
      set_outer_lanes(v.back());
      for (size_t k = 0; k < lv_.size(); ++k) {
        Level &L = lv_[k];
        L.rg = v[6 * k + 2];
        L.pg = v[6 * k + 3];
        set_layout(L, static_cast<int>(k), v[6 * k] != 0, v[6 * k + 1], ar_);
        L.coop = v[6 * k + 4] != 0 && opt_.sweep_launch != 0 && !L.relaxed && !opt_.half_sweeps;
        L.staged = v[6 * k + 5] != 0 && opt_.sweep_launch != 0 && block_ && L.sliced && L.g == 1 &&
                   prepare_staged<VT>(L.B.max_slots, device_);
      }
      return;
    }
  }
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), stream_));
  for (Level &L : lv_) {
    fill_kernel<VT><<<blocks_for(L.n, cap_blocks_), 256, 0, stream_>>>(L.n, L.x, VT(0));
    fill_kernel<VT><<<blocks_for(L.n, cap_blocks_), 256, 0, stream_>>>(L.n, L.b, VT(1));
    CKL("autotune fill");
  }
  for (size_t k = 0; k < lv_.size(); ++k) {
    Level &L = lv_[k];
    const bool coarsest_dense = k + 1 == lv_.size() && opt_.coarse == 1;
    if (!coarsest_dense) {
      float best = 1e30f;
      bool best_sliced = true;
      int bestg = 1;
      auto sweep = [&] { for (int c = 0; c < L.ncolors; ++c) gs_pass<VT>(L, c, L.b, L.x, false, stream_); };
      // sliced candidates with g > 1 are built into arenas of their own; the
      // fastest one's arena is kept (not rebuilt), the others are freed once
      // timed (time_ms waits for its launches)
      std::unique_ptr<Arena> best_arena;
      DevSell<VT> bestA;
      DevBell<VT> bestB;
      bool best_staged = false;
      for (int g : {1, 2, 4, 8}) {
        std::unique_ptr<Arena> trial(new Arena);
        set_layout(L, static_cast<int>(k), true, g, *trial);
        const float t = time_segment(sweep, 10);
        if (t < best) {
          best = t, best_sliced = true, bestg = g, best_staged = false;
          if (g > 1) best_arena = std::move(trial), bestA = L.A, bestB = L.B;
        }
        // block levels: BELL-1 also with the slices bulk-copied to shared memory
        if (g == 1 && block_ && opt_.sweep_launch == 1 && prepare_staged<VT>(L.B.max_slots, device_)) {
          L.staged = true;
          const float ts = time_segment(sweep, 10);
          L.staged = false;
          if (ts < best) best = ts, best_sliced = true, bestg = 1, best_staged = true;
        }
      }
      CK(cudaStreamSynchronize(stream_));
      set_layout(L, static_cast<int>(k), true, 1, ar_);
      for (int g : {4, 8, 16, 32}) {
        set_layout(L, static_cast<int>(k), false, g, ar_);
        const float t = time_segment(sweep, 10);
        if (t < best) best = t, best_sliced = false, bestg = g;
      }
      if (best_sliced && bestg > 1) {
        L.A = bestA;
        L.B = bestB;
        L.sliced = true;
        L.g = bestg;
        set_color_slices(L);
        kept_layouts_.push_back(std::move(best_arena));
      } else {
        set_layout(L, static_cast<int>(k), best_sliced, bestg, ar_);
      }
      L.staged = best_staged;
      // then one launch per colour pass against one cooperative launch per
      // symmetric step, on the chosen layout (the iterates are identical)
      // (half sweeps run one direction per smoothing call, as per-colour
      // passes: the cooperative step is never used there)
      if (L.kind == 0 && !block_ && !L.relaxed && !opt_.half_sweeps && opt_.sweep_launch == 1) {
        auto step = [&] { smooth<VT>(L, L.b, L.x, 1, false, stream_); };
        L.coop = false;
        const float t_pass = time_segment(step, 10);
        L.coop = true;
        float t_coop = 1e30f;
        try {
          t_coop = time_segment(step, 10);
          CgState hs{};
          CK(cudaMemcpy(&hs, st_, sizeof(CgState), cudaMemcpyDeviceToHost));
          check_sync_fault(hs);
        } catch (const CudaError &) {
          // a launch the device refused: close a capture left open, keep the
          // per-colour passes
          cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
          if (cudaStreamIsCapturing(stream_, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream_, &g);
            if (g != nullptr) cudaGraphDestroy(g);
          }
          cudaGetLastError();
          t_coop = 1e30f;
        }
        L.coop = t_coop < t_pass;
      }
    }
    if (k + 1 < lv_.size()) {
      Level &Cn = lv_[k + 1];
      // each candidate keeps the faster of two timings of its captured
      // launches: one timing alone can pick a slower layout when a clock or
      // cache transient hits the better candidate
      float bp = 1e30f, br = 1e30f;
      int gp = 1, gr = 1;
      for (int g : cands) {
        const float tr = time_segment([&] { transfer<kSpmvSet, VT>(L.R, L.Rc, g, L.x, Cn.b, (const VT *)nullptr, stream_); }, 10, 2);
        const float tp = time_segment([&] { transfer<kSpmvAdd, VT>(L.P, L.Pc, g, Cn.x, L.r, (const VT *)nullptr, stream_); }, 10, 2);
        if (tr < br) br = tr, gr = g;
        if (tp < bp) bp = tp, gp = g;
      }
      L.rg = gr;
      L.pg = gp;
    }
  }
  tune_outer();
  CKL("autotune");
  launches_ = 0;
  CK(cudaStreamSynchronize(stream_));
  if (!opt_.tune_cache.empty()) {
    std::ofstream out(opt_.tune_cache, std::ios::app);
    out << sig;
    for (const Level &L : lv_)
      out << " " << (L.sliced ? 1 : 0) << " " << L.g << " " << L.rg << " " << L.pg << " " << (L.coop ? 1 : 0) << " "
          << (L.staged ? 1 : 0);
    out << " " << (block_ ? cgB_.g : 1) << "\n";
  }
}

template <typename VT>
void AmgPcg<VT>::launch_tail(cudaStream_t s) {
  TailParams<VT> p;
  p.k0 = tail_k0_;
  p.L = static_cast<int>(lv_.size());
  p.pre = opt_.pre;
  p.post = opt_.post;
  p.coarse_steps = opt_.coarse_steps;
  p.coarse_dense = opt_.coarse == 1;
  p.alias = opt_.reference_vcycle;
  p.omega = VT(opt_.omega);
  p.lv = tail_lv_;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tail_cluster_, 1, 1);
  cfg.blockDim = dim3(1024, 1, 1);
  cfg.dynamicSmemBytes = tail_smem_;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = tail_cluster_;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int *done = &st_->done;
  CK(cudaLaunchKernelEx(&cfg, coarse_tail_kernel<VT>, p, done));
  CKL("coarse tail");
}

// Largest cluster of at most `want` CTAs (16, 8, 4, 2 or 1, 1024 threads
// each) the device co-schedules with `smem` bytes of dynamic shared memory
// per CTA; 0 if none.
template <typename VT>
int AmgPcg<VT>::tail_cluster_size(size_t smem, int want) {
  if (cudaFuncSetAttribute(coarse_tail_kernel<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int cand : {16, 8, 4, 2, 1}) {
    if (cand > want) continue;
    if (cand == 16 &&
        cudaFuncSetAttribute(coarse_tail_kernel<VT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cand, 1, 1);
    cfg.blockDim = dim3(1024, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cand;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, coarse_tail_kernel<VT>, &cfg) == cudaSuccess && nclusters >= 1)
      return cand;
    cudaGetLastError();
  }
  return 0;
}

// Level table of a tail starting at k0: x replicas packed in shared memory
// (each level's replica 16-byte aligned).
template <typename VT>
void AmgPcg<VT>::upload_tail_table(int k0) {
  const int L = static_cast<int>(lv_.size());
  std::vector<TailLevel<VT>> hl(L);
  auto lanes = [](int g) { return g < 4 ? 4 : g; };
  const int align = 16 / static_cast<int>(sizeof(VT));
  int off = 0;
  for (int k = k0; k < L; ++k) {
    Level &lv = lv_[k];
    TailLevel<VT> &t = hl[k];
    t.n = lv.n;
    t.ncolors = lv.ncolors;
    t.g = lanes(lv.g);
    t.xoff = off;
    off += (lv.n + align - 1) / align * align;
    t.color_first = ar_.upload(lv.color_first);
    t.wts = lv.wts.empty() || lv.wts[0] == nullptr ? nullptr : lv.wts[0];
    t.A = lv.C.view();
    if (k + 1 < L) {
      t.R = lv.Rc.view();
      t.P = lv.Pc.view();
      t.rg = lanes(lv.rg);
      t.pg = lanes(lv.pg);
    }
    t.x = lv.x;
    t.b = lv.b;
    t.r = lv.r;
    t.ainv = lv.ainv;
  }
  if (tail_lv_ == nullptr) tail_lv_ = ar_.alloc<TailLevel<VT>>(L);
  CK(cudaMemcpy(tail_lv_, hl.data(), sizeof(TailLevel<VT>) * L, cudaMemcpyHostToDevice));
  tail_smem_ = static_cast<size_t>(off) * sizeof(VT);
  tail_k0_ = k0;
}

// Times f() as the solve will run it: replayed from a captured CUDA graph
// in graph mode, launched on the stream otherwise.
template <typename VT>
float AmgPcg<VT>::time_segment(const std::function<void()> &f, int reps, int trials) {
  if (!opt_.graph) {
    float t = time_ms(f, reps);
    for (int i = 1; i < trials; ++i) t = std::min(t, time_ms(f, reps));
    return t;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t e = nullptr;
  {
    const PlainLaunches plain(pdl_, opt_.overlap_launch == 2);
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    f();
    CK(cudaStreamEndCapture(stream_, &g));
  }
  CK(cudaGraphInstantiate(&e, g, 0));
  float t = time_ms([&] { CK(cudaGraphLaunch(e, stream_)); }, reps);
  for (int i = 1; i < trials; ++i) t = std::min(t, time_ms([&] { CK(cudaGraphLaunch(e, stream_)); }, reps));
  CK(cudaGraphExecDestroy(e));
  CK(cudaGraphDestroy(g));
  return t;
}

// Picks where the cluster-resident tail starts and how many CTAs it uses.
// Candidate start levels are k >= 1 whose replicas (levels k..L-1) fit in
// 200 KB of shared memory; candidate clusters have 16, 8, 4, 2 or 1 CTAs
// (small levels are bound by the barrier, large ones by the loads). Every
// candidate, and no tail at all, runs the V-cycle from the smallest
// candidate level on the same inputs, timed the way the solve runs it
// (graph replay in graph mode); the fastest configuration is kept. A forced
// tail (tail == 2) starts at the smallest candidate level.
template <typename VT>
void AmgPcg<VT>::setup_tail() {
  tail_on_ = false;
  const int L = static_cast<int>(lv_.size());
  if (opt_.tail == 0 || L < 2) return;
  // The tail reads only the full row-major inverse, and one cluster of <= 16
  // SMs streaming a large one cannot keep up with a launch over all SMs.
  if (opt_.coarse == 1 && (lv_[L - 1].packed || lv_[L - 1].n > 8192)) return;
  const size_t budget = 200 * 1024;
  std::vector<int> cands;
  size_t bytes = 0;
  for (int k = L - 1; k >= 1; --k) {
    bytes += (static_cast<size_t>(lv_[k].n) + 4) * sizeof(VT);
    if (bytes > budget || lv_[k].n > opt_.tail_rows) break;
    cands.push_back(k);
  }
  if (cands.empty()) return;
  const int kmin = cands.back();
  // a recorded decision for this hierarchy ("tail:<signature> k0 cluster", k0 -1 = no tail)
  const std::string key = "tail:" + signature();
  if (opt_.tail == 1 && !opt_.tune_cache.empty()) {
    std::ifstream in(opt_.tune_cache);
    std::string line, k;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      int k0 = -1, cl = 0;
      ls >> k >> k0 >> cl;
      if (!ls || k != key) continue;
      if (k0 >= 0 && std::find(cands.begin(), cands.end(), k0) != cands.end()) {
        upload_tail_table(k0);
        if (tail_cluster_size(tail_smem_, cl) == cl) {  // also applies the function attributes
          tail_cluster_ = cl;
          tail_on_ = true;
        }
      }
      if (!tail_on_) tail_k0_ = -1;
      return;
    }
  }
  Level &T0 = lv_[kmin];
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), stream_));
  fill_kernel<VT><<<blocks_for(T0.n, cap_blocks_), 256, 0, stream_>>>(T0.n, T0.b, VT(1));
  CKL("tail timing fill");
  auto segment = [&] { vcycle<VT>(kmin, T0.b, T0.x, true, stream_); };
  float best = 1e30f;
  int best_k0 = -1, best_cl = 0;
  if (opt_.tail == 1) best = time_segment(segment, 3);
  for (int k0 : cands) {
    if (opt_.tail == 2 && k0 != kmin) continue;
    upload_tail_table(k0);
    int prev = 0;
    for (int want : {16, 8, 4, 2, 1}) {
      const int cl = tail_cluster_size(tail_smem_, want);
      if (cl == 0 || cl == prev) continue;
      prev = cl;
      tail_cluster_ = cl;
      tail_on_ = true;
      const float t = time_segment(segment, 3);
      tail_on_ = false;
      if (t < best || (opt_.tail == 2 && best_k0 < 0)) best = t, best_k0 = k0, best_cl = cl;
    }
  }
  if (best_k0 >= 0) {
    upload_tail_table(best_k0);
    tail_cluster_ = best_cl;
    tail_cluster_size(tail_smem_, best_cl);  // re-applies the function attributes
    tail_on_ = true;
  }
  if (!tail_on_) tail_k0_ = -1;
  launches_ = 0;
  CK(cudaStreamSynchronize(stream_));
  if (opt_.tail == 1 && !opt_.tune_cache.empty()) {
    std::ofstream out(opt_.tune_cache, std::ios::app);
    out << key << " " << (tail_on_ ? tail_k0_ : -1) << " " << (tail_on_ ? tail_cluster_ : 0) << "\n";
  }
}

// Multigrid*Preconditioner::apply: z = 0, then `vcycles` V-cycles.
template <typename VT>
void AmgPcg<VT>::precondition(const double *r, VT *z, cudaStream_t s) {
  for (int v = 0; v < opt_.vcycles; ++v) vcycle<double>(0, r, z, v == 0, s);
}

// The outer 3x3 block operator in BELL-32 with g lanes per node (rebuilt
// from the finest level's host matrix; the previous copy is freed).
template <typename VT>
void AmgPcg<VT>::set_outer_lanes(int g) {
  if (!block_ || g == cgB_.g) return;
  if (g != 1 && g != 2 && g != 4 && g != 8) throw std::runtime_error("tune cache: bad lanes of the outer operator");
  std::unique_ptr<Arena> a(new Arena);
  cgB_ = upload_bell(*a, make_bell<double>(host_A_.at(0), lv_[0].color_first, g));
  cg_arena_ = std::move(a);
}

// Lanes per node of the outer block operator: 1, 2, 4 and 8 each run the
// FP64 SpMV + p.Ap kernel 10 times (graph-replayed in graph mode) on p = 1;
// the fastest layout is kept, the others are freed.
template <typename VT>
void AmgPcg<VT>::tune_outer() {
  if (!block_) return;
  fill_kernel<double><<<blocks_for(n0_, cap_blocks_), 256, 0, stream_>>>(n0_, p_, 1.0);
  CKL("autotune fill");
  CgState init{};
  init.rho = 1.0;
  const DevBell<double> base = cgB_;
  DevBell<double> best = base;
  std::unique_ptr<Arena> best_arena;
  float tbest = 1e30f;
  for (int g : {1, 2, 4, 8}) {
    std::unique_ptr<Arena> trial;
    if (g == base.g) {
      cgB_ = base;
    } else {
      trial.reset(new Arena);
      cgB_ = upload_bell(*trial, make_bell<double>(host_A_.at(0), lv_[0].color_first, g));
    }
    CK(cudaMemcpyAsync(scratch_st_, &init, sizeof(CgState), cudaMemcpyHostToDevice, stream_));
    const float t = time_segment([&] { outer_spmv(p_, scratch_st_, stream_); }, 10);
    if (t < tbest) {
      tbest = t;
      best = cgB_;
      best_arena = std::move(trial);  // null for the base copy
    }
  }
  CK(cudaStreamSynchronize(stream_));
  cgB_ = best;
  if (best.g != base.g) cg_arena_ = std::move(best_arena);
}

// The outer FP64 operator: ap = A v and v.Ap (alpha) into `st`.
template <typename VT>
void AmgPcg<VT>::outer_spmv(const double *v, CgState *st, cudaStream_t s) {
  if (!block_) {
    cg_spmv_pap_kernel<<<blocks_for(32LL * cgA_.nslices, cap_blocks_), 256, 0, s>>>(cgA_.view(), v, ap_, st, partials_);
    return;
  }
  const int blocks = blocks_for(32LL * cgB_.nslices, cap_blocks_);
  switch (cgB_.g) {
    case 1: cg_bell_spmv_pap_kernel<1><<<blocks, 256, 0, s>>>(cgB_.view(), v, ap_, st, partials_); break;
    case 2: cg_bell_spmv_pap_kernel<2><<<blocks, 256, 0, s>>>(cgB_.view(), v, ap_, st, partials_); break;
    case 4: cg_bell_spmv_pap_kernel<4><<<blocks, 256, 0, s>>>(cgB_.view(), v, ap_, st, partials_); break;
    default: cg_bell_spmv_pap_kernel<8><<<blocks, 256, 0, s>>>(cgB_.view(), v, ap_, st, partials_); break;
  }
}

// r = b - A x with the outer FP64 operator.
template <typename VT>
void AmgPcg<VT>::outer_resid(cudaStream_t s) {
  if (!block_) {
    sell_spmv_kernel<double, double, kSpmvResid>
        <<<blocks_for(32LL * cgA_.nslices, cap_blocks_), 256, 0, s>>>(cgA_.view(), x_, r_, b_, nullptr);
    return;
  }
  const int blocks = blocks_for(32LL * cgB_.nslices, cap_blocks_);
  switch (cgB_.g) {
    case 1: bell_spmv_kernel<double, double, kSpmvResid, 1><<<blocks, 256, 0, s>>>(cgB_.view(), x_, r_, b_, nullptr); break;
    case 2: bell_spmv_kernel<double, double, kSpmvResid, 2><<<blocks, 256, 0, s>>>(cgB_.view(), x_, r_, b_, nullptr); break;
    case 4: bell_spmv_kernel<double, double, kSpmvResid, 4><<<blocks, 256, 0, s>>>(cgB_.view(), x_, r_, b_, nullptr); break;
    default: bell_spmv_kernel<double, double, kSpmvResid, 8><<<blocks, 256, 0, s>>>(cgB_.view(), x_, r_, b_, nullptr); break;
  }
}

template <typename VT>
void AmgPcg<VT>::cg_iteration(int parity, cudaStream_t s) {
  VT *z_old = z_[parity], *z_new = z_[parity ^ 1];
  outer_spmv(p_, st_, s);
  CKL("cg spmv");
  cg_update_xr_kernel<<<blocks_for(n0_, cap_blocks_), 256, 0, s>>>(n0_, x_, r_, p_, ap_, st_, partials_);
  CKL("cg update");
  precondition(r_, z_new, s);
  cg_dot_rz_kernel<VT><<<blocks_for(n0_, cap_blocks_), 256, 0, s>>>(n0_, r_, z_new, opt_.flexible ? z_old : nullptr, st_, partials_);
  CKL("cg dot");
  cg_update_p_kernel<VT><<<blocks_for(n0_, cap_blocks_), 256, 0, s>>>(n0_, z_new, p_, st_);
  CKL("cg p update");
}

// r = b - A x; z = M r; p = z; bb, rho, rr.
template <typename VT>
void AmgPcg<VT>::cg_start(cudaStream_t s) {
  CgState init{};
  init.tol2 = opt_.tol * opt_.tol;
  init.max_iter = opt_.max_iter;
  init.flexible = opt_.flexible;
  // pageable source: staged by the runtime before the call returns
  CK(cudaMemcpyAsync(st_, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  outer_resid(s);
  CKL("initial residual");
  precondition(r_, z_[0], s);
  cg_init_kernel<VT><<<blocks_for(n0_, cap_blocks_), 256, 0, s>>>(n0_, b_, r_, z_[0], p_, st_, partials_);
  CKL("cg init");
}

template <typename VT>
void AmgPcg<VT>::ensure_graphs() {
  if (exec_[0] != nullptr) return;
  for (int par = 0; par < 2; ++par) {
    const long long before = launches_;
    {
      const PlainLaunches plain(pdl_, opt_.overlap_launch == 2);
      CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      cg_iteration(par, stream_);
      CK(cudaStreamEndCapture(stream_, &graph_[par]));
    }
    CK(cudaGraphInstantiate(&exec_[par], graph_[par], 0));
    graph_kernels_ = launches_ - before;
    launches_ = before;  // captured, not executed
  }
}

template <typename VT>
void AmgPcg<VT>::run(cudaStream_t user, SolveStats *out) {
  // Order after the caller's stream, work on the solver's own stream.
  CK(cudaEventRecord(ev_[0], user));
  CK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  CK(cudaEventRecord(ev_[2], stream_));
  cg_start(stream_);
  CK(cudaMemcpyAsync(&host_st_[0], st_, sizeof(CgState), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  CgState hs = host_st_[0];
  int spmv = 0;
  if (!(std::sqrt(hs.bb) >= 1e-12)) {
    // CGSolver::solve: a zero right-hand side returns x = 0.
    if (std::isfinite(hs.bb)) {
      CK(cudaMemsetAsync(x_, 0, sizeof(double) * n0_, stream_));
      hs.status = kCgZeroRhs;
      hs.iterations = 0;
    }
  } else if (!hs.done) {
    if (opt_.graph) {
      ensure_graphs();
      // Keep one iteration queued ahead of the host check; kernels of an
      // iteration queued after the stop flag was set return immediately.
      int it = 0;
      for (; it < opt_.max_iter; ++it) {
        CK(cudaGraphLaunch(exec_[it & 1], stream_));
        launches_ += graph_kernels_;
        CK(cudaMemcpyAsync(&host_st_[it & 1], st_, sizeof(CgState), cudaMemcpyDeviceToHost, stream_));
        CK(cudaEventRecord(ev_[it & 1], stream_));
        if (it >= 1) {
          CK(cudaEventSynchronize(ev_[(it - 1) & 1]));
          if (host_st_[(it - 1) & 1].done) break;
        }
      }
      CK(cudaStreamSynchronize(stream_));
      CK(cudaMemcpy(&host_st_[0], st_, sizeof(CgState), cudaMemcpyDeviceToHost));
      hs = host_st_[0];
    } else {
      // CGSolver::solve: one submitAndWait and one scalar read per iteration.
      for (int it = 0; it < opt_.max_iter; ++it) {
        cg_iteration(it & 1, stream_);
        CK(cudaMemcpyAsync(&host_st_[0], st_, sizeof(CgState), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (host_st_[0].done) break;
      }
      hs = host_st_[0];
    }
    spmv = hs.iter;
  }
  CK(cudaEventRecord(ev_[3], stream_));
  CK(cudaEventRecord(ev_[1], stream_));
  CK(cudaStreamWaitEvent(user, ev_[1], 0));
  CK(cudaEventSynchronize(ev_[3]));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
  check_sync_fault(hs);
  if (out != nullptr) {
    out->iterations = hs.iterations;
    out->status = hs.status;
    out->ratio = hs.ratio;
    out->bb = hs.bb;
    out->spmv = spmv;
    out->solve_ms = ms;
  }
  if (hs.status == kCgNotFinite)
    throw std::runtime_error("CGSolver: solver diverged (NaN/Inf residual).");
}

template <typename VT>
void AmgPcg<VT>::solve_device(const double *b, double *x, cudaStream_t stream, SolveStats *st) {
  CK(cudaSetDevice(device_));
  CK(cudaEventRecord(ev_[0], stream));
  CK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  const int blocks = blocks_for(n0_, cap_blocks_);
  scatter_kernel<double, double><<<blocks, 256, 0, stream_>>>(n0_, q0_, b, b_);
  scatter_kernel<double, double><<<blocks, 256, 0, stream_>>>(n0_, q0_, x, x_);
  CKL("permute in");
  ++launches_;
  CK(cudaEventRecord(ev_[1], stream_));
  CK(cudaStreamWaitEvent(stream, ev_[1], 0));
  run(stream, st);
  CK(cudaEventRecord(ev_[0], stream));
  CK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  gather_kernel<double, double><<<blocks, 256, 0, stream_>>>(n0_, q0_, x_, x);
  CKL("permute out");
  CK(cudaEventRecord(ev_[1], stream_));
  CK(cudaStreamWaitEvent(stream, ev_[1], 0));
  CK(cudaStreamSynchronize(stream));
}

template <typename VT>
void AmgPcg<VT>::solve_host(const double *b, double *x, SolveStats *st) {
  CK(cudaSetDevice(device_));
  CK(cudaMemcpyAsync(ubuf_, b, sizeof(double) * n0_, cudaMemcpyHostToDevice, stream_));
  CK(cudaMemcpyAsync(uxbuf_, x, sizeof(double) * n0_, cudaMemcpyHostToDevice, stream_));
  solve_device(ubuf_, uxbuf_, stream_, st);
  CK(cudaMemcpyAsync(x, uxbuf_, sizeof(double) * n0_, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
}

template <typename VT>
void AmgPcg<VT>::apply_preconditioner(const double *r, double *z, cudaStream_t stream) {
  CK(cudaSetDevice(device_));
  CK(cudaEventRecord(ev_[0], stream));
  CK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), stream_));  // clears the stop flag
  const int blocks = blocks_for(n0_, cap_blocks_);
  scatter_kernel<double, double><<<blocks, 256, 0, stream_>>>(n0_, q0_, r, r_);
  precondition(r_, z_[0], stream_);
  gather_kernel<VT, double><<<blocks, 256, 0, stream_>>>(n0_, q0_, z_[0], z);
  CKL("apply preconditioner");
  ++launches_;  // the scatter before the V-cycle
  CK(cudaEventRecord(ev_[1], stream_));
  CK(cudaStreamWaitEvent(stream, ev_[1], 0));
  CK(cudaStreamSynchronize(stream));
}

template <typename VT>
double AmgPcg<VT>::time_level(int level, int op, int lanes, int reps, cudaStream_t stream) {
  if (level < 0 || level + 1 >= static_cast<int>(lv_.size()))
    throw std::runtime_error("time_level: level must have a coarser level below it");
  if (op < 0 || op > 3) throw std::runtime_error("time_level: op must be 0, 1, 2 or 3");
  if (lanes != 0 && lanes != 1 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    throw std::runtime_error("time_level: lanes must be 0, 1, 4, 8, 16 or 32");
  CK(cudaSetDevice(device_));
  if (reps < 1) reps = 1;
  // graph capture is not possible on the legacy default stream
  if (opt_.graph && stream == nullptr) stream = stream_;
  Level &L = lv_[level];
  Level &C = lv_[level + 1];
  const int sg = L.g, spg = L.pg, srg = L.rg;
  const bool ssl = L.sliced, scoop = L.coop, sstaged = L.staged;
  const DevSell<VT> sA = L.A;
  const DevBell<VT> sB = L.B;
  const std::vector<int> scs = L.color_slice;
  auto restore = [&] {
    L.g = sg, L.pg = spg, L.rg = srg, L.sliced = ssl, L.A = sA, L.B = sB, L.coop = scoop, L.staged = sstaged;
    if (L.color_slice != scs) {
      L.color_slice = scs;
      CK(cudaMemcpy(L.d_color_slice, scs.data(), sizeof(int) * scs.size(), cudaMemcpyHostToDevice));
    }
  };
  if (lanes != 0) {
    if (op <= 1) {
      L.coop = false;  // a forced layout runs its per-colour passes
      L.staged = false;
      L.sliced = lanes == 1;
      L.g = lanes;
      if (lanes == 1) {
        L.A = L.A1;
        L.B = L.B1;
        set_color_slices(L);
      }
    } else if (op == 2) {
      L.rg = lanes;
    } else {
      L.pg = lanes;
    }
  }
  const long long saved = launches_;
  auto launch = [&]() {
    if (op == 0) {
      forward_sweep(L, stream);
    } else if (op == 1) {
      level_spmv_resid<VT>(L, L.b, L.x, L.r, stream);
    } else if (op == 2) {
      transfer<kSpmvSet, VT>(L.R, L.Rc, L.rg, L.r, C.b, (const VT *)nullptr, stream);
    } else {
      transfer<kSpmvAdd, VT>(L.P, L.Pc, L.pg, C.x, L.x, (const VT *)nullptr, stream);
    }
  };
  // defined inputs: x = 0, b = 1 on both levels; the stop flag cleared
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), stream));
  for (Level *l : {&L, &C}) {
    fill_kernel<VT><<<blocks_for(l->n, cap_blocks_), 256, 0, stream>>>(l->n, l->x, VT(0));
    fill_kernel<VT><<<blocks_for(l->n, cap_blocks_), 256, 0, stream>>>(l->n, l->b, VT(1));
  }
  float ms = 0.f;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  try {
    launch();
    launch();
    CKL("time_level warm-up");
    if (opt_.graph) {
      // as the solve runs it: the repetitions replayed from one captured graph
      {
        const PlainLaunches plain(pdl_, opt_.overlap_launch == 2);
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < reps; ++i) launch();
        CK(cudaStreamEndCapture(stream, &graph));
      }
      CK(cudaGraphInstantiate(&exec, graph, 0));
      CK(cudaGraphLaunch(exec, stream));
      CK(cudaEventRecord(ev_[2], stream));
      CK(cudaGraphLaunch(exec, stream));
      CK(cudaEventRecord(ev_[3], stream));
    } else {
      CK(cudaEventRecord(ev_[2], stream));
      for (int i = 0; i < reps; ++i) launch();
      CK(cudaEventRecord(ev_[3], stream));
    }
    CK(cudaEventSynchronize(ev_[3]));
    CK(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
    if (exec) cudaGraphExecDestroy(exec), exec = nullptr;
    if (graph) cudaGraphDestroy(graph), graph = nullptr;
    CgState hs{};
    CK(cudaMemcpy(&hs, st_, sizeof(CgState), cudaMemcpyDeviceToHost));
    check_sync_fault(hs);
  } catch (...) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g != nullptr) cudaGraphDestroy(g);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    restore();
    throw;
  }
  restore();
  launches_ = saved;
  return ms / reps;
}

template <typename VT>
double AmgPcg<VT>::time_kernel(int kind, int reps, cudaStream_t stream) {
  CK(cudaSetDevice(device_));
  if (reps < 1) reps = 1;
  CgState s{};
  s.rho = 1.0;
  CK(cudaMemcpyAsync(scratch_st_, &s, sizeof(CgState), cudaMemcpyHostToDevice, stream));
  Level &L = lv_[0];
  auto launch = [&]() {
    if (kind == 0) {
      outer_spmv(p_, scratch_st_, stream);
    } else if (kind == 1) {
      // exactly the solve's launch path (format and launch mode chosen by the autotuner)
      forward_sweep(L, stream);
    } else if (kind == 2) {
      level_spmv_resid<VT>(L, L.b, L.x, L.r, stream);
    } else {
      Level &Cl = lv_.back();
      dense_coarse<VT>(Cl, Cl.b, Cl.x, stream);
    }
  };
  if (kind < 0 || kind > 3) throw std::runtime_error("time_kernel: kind must be 0..3");
  if (kind == 3 && (opt_.coarse != 1 || (lv_.back().ainv == nullptr && lv_.back().ainv_h == nullptr)))
    throw std::runtime_error("time_kernel: the solver has no dense coarsest solve");
  // defined inputs: p = 1, level-0 x = 0, b = 1; the stop flag cleared
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), stream));
  fill_kernel<double><<<blocks_for(n0_, cap_blocks_), 256, 0, stream>>>(n0_, p_, 1.0);
  fill_kernel<VT><<<blocks_for(L.n, cap_blocks_), 256, 0, stream>>>(L.n, L.x, VT(0));
  fill_kernel<VT><<<blocks_for(L.n, cap_blocks_), 256, 0, stream>>>(L.n, L.b, VT(1));
  {
    Level &Cl = lv_.back();
    fill_kernel<VT><<<blocks_for(Cl.n, cap_blocks_), 256, 0, stream>>>(Cl.n, Cl.b, VT(1));
  }
  launch();
  launch();
  CKL("time_kernel warm-up");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, stream));
  for (int i = 0; i < reps; ++i) launch();
  CK(cudaEventRecord(e1, stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CKL("time_kernel");
  CgState hs{};
  CK(cudaMemcpy(&hs, st_, sizeof(CgState), cudaMemcpyDeviceToHost));
  check_sync_fault(hs);
  return ms / reps;
}

template <typename VT>
double AmgPcg<VT>::error_reduction(const double *e0, cudaStream_t stream) {
  CK(cudaSetDevice(device_));
  CK(cudaEventRecord(ev_[0], stream));
  CK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  cudaStream_t s = stream_;
  const int blocks = blocks_for(n0_, cap_blocks_);
  CgState init{};
  init.rho = 1.0;
  CK(cudaMemcpyAsync(scratch_st_, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(st_, 0, sizeof(CgState), s));  // clears the stop flag of the V-cycle kernels
  scatter_kernel<double, double><<<blocks, 256, 0, s>>>(n0_, q0_, e0, x_);
  auto energy = [&](const double *v) {
    outer_spmv(v, scratch_st_, s);
    CKL("energy");
    CgState h{};
    CK(cudaMemcpyAsync(&h, scratch_st_, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h.pAp;
  };
  const double e0a = energy(x_);           // ap_ = A e0
  precondition(ap_, z_[0], s);             // z = M A e0
  sub_kernel<VT><<<blocks, 256, 0, s>>>(n0_, x_, z_[0], p_);  // e1 = e0 - z
  CKL("error update");
  const double e1a = energy(p_);
  if (!(e0a > 0.0)) throw std::runtime_error("error_reduction: e0 has zero energy");
  return std::sqrt(std::max(e1a, 0.0) / e0a);
}

}  // namespace

std::unique_ptr<Solver> Solver::create(const Hierarchy &h, const std::vector<const int *> &o2n,
                                       const std::vector<const int *> &n2o,
                                       const SolverOptions &opt, int device) {
  if (opt.mixed) return std::unique_ptr<Solver>(new AmgPcg<float>(h, o2n, n2o, opt, device));
  return std::unique_ptr<Solver>(new AmgPcg<double>(h, o2n, n2o, opt, device));
}

}  // namespace gsb
