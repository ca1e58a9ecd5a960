// Batched AMG-PCG: setup (per-system colouring and colour-contiguous order,
// the batch layout, work lists, the threads-per-row autotuner) and the launch
// sequence of one CG iteration over every system, replayed as a CUDA graph.
//
// Schedule of one V-cycle over the batch. Level k of the batch holds every
// system with more than k levels; a system is "smoothed" on level k when k is
// not its coarsest level. Going down, level k is pre-smoothed, its residual
// formed and restricted to level k + 1 for the smoothed systems; at the
// bottom every system solves its own coarsest level (wherever that is) with
// its dense inverse in one launch; going up, each level receives the
// prolongated correction and is post-smoothed. Each system therefore sees
// exactly the order of operations of its own V-cycle
// (src/Smoothers/MultigridSmoother.cc:337-412), while a launch carries the
// same step of all systems.
#include "batch.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <thread>

#include "batch.cuh"
#include "dense.h"
#include "formats.cuh"

namespace gsb {

namespace {

#define BCK(x) cuda_check((x), #x)

constexpr int kSellItemSlices = 8;  // GS / SpMV items: one slice per warp of a 256-thread block
constexpr int kCgItemSlices = 32;   // CG items: up to 1024 rows, one partial sum each
constexpr int kCsrvTrips = 1;       // CSR-vector items: 256 / G rows, one trip (coarse passes are latency-bound)
constexpr int kDenseItemRows = 32;  // coarsest-level items: 32 rows of one system

// Rows [r0, r1) of one system on one batch level; c0 = first row of their colour.
struct Seg {
  int sys, r0, r1, c0;
};

struct SysLevel {
  Csr A;                // internal (colour-contiguous) order
  std::vector<int> cf;  // colour offsets
  Csr P, R;             // P: this level <- next, R: next <- this; empty on the coarsest
};

struct SysPrep {
  std::vector<SysLevel> lv;
  std::vector<int> q0;       // internal index of caller row i on level 0
  std::vector<double> ainv;  // dense inverse of the coarsest level, internal order
};

// One system: greedy colouring of every level in natural order
// (src/Smoothers/SymmetricGaussSeidelSmoother.cc:33-43 with identity
// permutations) and the colour-contiguous relabelling of A, P and R.
SysPrep prepare_system(const Hierarchy &h, int levels_used, int coloring) {
  if (static_cast<int>(h.P.size()) + 1 != static_cast<int>(h.A.size()) ||
      static_cast<int>(h.R.size()) + 1 != static_cast<int>(h.A.size()))
    throw std::runtime_error("MultigridSmoother: invalid number of transfers.");
  const int L = std::min(levels_used, static_cast<int>(h.A.size()));
  if (L < 2)
    throw std::runtime_error("batched solver: every system needs at least two levels "
                             "(a system of at most min_dofs rows is a single dense solve)");
  if (h.block != 1) throw std::runtime_error("batched solver: scalar systems only (block size 1)");
  SysPrep sp;
  sp.lv.resize(L);
  std::vector<std::vector<int>> Q(L);
  for (int k = 0; k < L; ++k) {
    const Csr &Ak = h.A[k];
    Ak.check("hierarchy level matrix");
    if (Ak.rows != Ak.cols) throw std::runtime_error("level matrix must be square");
    std::vector<int> colors, verts, offs;
    if (coloring == 1) smallest_last_coloring(Ak.rows, Ak.rp.data(), Ak.ci.data(), colors, verts, offs);
    else greedy_coloring(Ak.rows, Ak.rp.data(), Ak.ci.data(), colors, verts, offs);
    Q[k].resize(Ak.rows);
    for (size_t i = 0; i < verts.size(); ++i) Q[k][verts[i]] = static_cast<int>(i);
    SysLevel &lv = sp.lv[k];
    lv.A = permute_matrix(Ak, Q[k].data(), Q[k].data());
    lv.cf = offs;
    for (int r = 0; r < lv.A.rows; ++r) {
      bool found = false;
      for (int e = lv.A.rp[r]; e < lv.A.rp[r + 1]; ++e)
        if (lv.A.ci[e] == r && std::fabs(lv.A.v[e]) >= 1e-12) found = true;
      if (!found) throw std::runtime_error("Gauss-Seidel: zero or missing diagonal entry.");
    }
    if (k > 0) {
      SysLevel &f = sp.lv[k - 1];
      f.P = permute_matrix(h.P[k - 1], Q[k - 1].data(), Q[k].data());
      f.R = permute_matrix(h.R[k - 1], Q[k].data(), Q[k - 1].data());
      if (f.P.rows != f.A.rows || f.P.cols != Ak.rows || f.R.rows != Ak.rows || f.R.cols != f.A.rows)
        throw std::runtime_error("MultigridSmoother: transfer operator shape mismatch.");
    }
  }
  sp.q0 = Q[0];
  return sp;
}

// All systems, several at a time (the host dense inverses dominate). The
// levels used follow the dense-coarsest rule of dense_depth: with
// coarse_rows > 0 every system stops at min(own depth, D), D the deepest
// "first level with at most coarse_rows rows" over the systems, so whole
// batch levels (and their launches) drop out. Coarsest levels above
// kHostInverseRows rows are left for the GPU inverse.
std::vector<SysPrep> prepare_all(const std::vector<const Hierarchy *> &h, bool with_inverse, int coarse_rows,
                                 int coloring) {
  const int S = static_cast<int>(h.size());
  int D = 0;
  for (int i = 0; i < S; ++i) {
    if (h[i] == nullptr) throw std::runtime_error("batched solver: null hierarchy");
    std::vector<int> rows;
    for (const Csr &a : h[i]->A) rows.push_back(a.rows);
    D = std::max(D, dense_depth(rows, coarse_rows));
  }
  std::vector<SysPrep> out(S);
  std::vector<std::string> err(S);
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int i; (i = next++) < S;) {
      try {
        out[i] = prepare_system(*h[i], D, coloring);
        if (with_inverse && out[i].lv.back().A.rows <= kHostInverseRows)
          out[i].ainv = cholesky_inverse(out[i].lv.back().A);
      } catch (const std::exception &e) {
        err[i] = e.what();
      }
    }
  };
  const int nt = std::max(1, std::min<int>(S, host_threads()));
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto &t : th) t.join();
  for (int i = 0; i < S; ++i)
    if (!err[i].empty()) throw std::runtime_error("system " + std::to_string(i) + ": " + err[i]);
  return out;
}

struct Layout {
  int S = 0, K = 0;
  std::vector<int> L;                                  // levels per system
  std::vector<std::vector<int>> off;                   // [k][s] first row, -1 absent
  std::vector<int> rows;                               // [k]
  std::vector<int> maxc;                               // [k] colour passes per sweep
  std::vector<std::vector<std::vector<Seg>>> fwd, bwd; // [k][pass]
  std::vector<std::vector<Seg>> whole;                 // [k] smoothed systems, all their rows
  std::vector<std::vector<Seg>> below;                 // [k] systems on level k + 1, their rows there
  std::vector<std::vector<int>> bounds;                // [k] system and colour boundaries
  std::vector<std::vector<int>> sys_bounds;            // [k] system boundaries
};

Layout make_layout(const std::vector<SysPrep> &sp) {
  Layout ly;
  ly.S = static_cast<int>(sp.size());
  for (const SysPrep &p : sp) {
    ly.L.push_back(static_cast<int>(p.lv.size()));
    ly.K = std::max(ly.K, ly.L.back());
  }
  const int K = ly.K, S = ly.S;
  ly.off.assign(K, std::vector<int>(S, -1));
  ly.rows.assign(K, 0);
  ly.maxc.assign(K, 0);
  ly.fwd.resize(K);
  ly.bwd.resize(K);
  ly.whole.resize(K);
  ly.below.resize(K);
  ly.bounds.resize(K);
  ly.sys_bounds.resize(K);
  for (int k = 0; k < K; ++k) {
    long long r = 0;
    for (int s = 0; s < S; ++s) {
      if (ly.L[s] <= k) continue;
      ly.off[k][s] = static_cast<int>(r);
      r += sp[s].lv[k].A.rows;
      if (r > (1LL << 30)) throw std::runtime_error("batched solver: too many rows on one level");
    }
    ly.rows[k] = static_cast<int>(r);
  }
  for (int k = 0; k < K; ++k) {
    std::vector<int> &bd = ly.bounds[k], &sb = ly.sys_bounds[k];
    bd.push_back(0);
    sb.push_back(0);
    for (int s = 0; s < S; ++s) {
      if (ly.L[s] <= k) continue;
      const SysLevel &lv = sp[s].lv[k];
      const int o = ly.off[k][s], C = static_cast<int>(lv.cf.size()) - 1;
      for (int c = 0; c <= C; ++c) bd.push_back(o + lv.cf[c]);
      sb.push_back(o + lv.A.rows);
      if (ly.L[s] - 1 > k) {  // smoothed on this level
        ly.maxc[k] = std::max(ly.maxc[k], C);
        ly.whole[k].push_back(Seg{s, o, o + lv.A.rows, o});
      }
    }
    std::sort(bd.begin(), bd.end());
    bd.erase(std::unique(bd.begin(), bd.end()), bd.end());
    ly.fwd[k].resize(ly.maxc[k]);
    ly.bwd[k].resize(ly.maxc[k]);
    for (int s = 0; s < S; ++s) {
      if (ly.L[s] - 1 <= k) continue;
      const SysLevel &lv = sp[s].lv[k];
      const int o = ly.off[k][s], C = static_cast<int>(lv.cf.size()) - 1;
      for (int c = 0; c < C; ++c) {
        const Seg g{s, o + lv.cf[c], o + lv.cf[c + 1], o + lv.cf[c]};
        if (g.r1 <= g.r0) continue;
        ly.fwd[k][c].push_back(g);
        ly.bwd[k][C - 1 - c].push_back(g);
      }
      if (k + 1 < K) {
        const int oc = ly.off[k + 1][s];
        ly.below[k].push_back(Seg{s, oc, oc + sp[s].lv[k + 1].A.rows, oc});
      }
    }
  }
  return ly;
}

// Slice starts of SELL-32 over `bounds` (as make_sell cuts them).
std::vector<int> slice_rows(const std::vector<int> &bounds, int rows) {
  std::vector<int> srow;
  for (size_t b = 0; b + 1 < bounds.size(); ++b)
    for (int r = bounds[b]; r < bounds[b + 1]; r += 32) srow.push_back(r);
  srow.push_back(rows);
  return srow;
}

void sell_items(const std::vector<Seg> &segs, const std::vector<int> &srow, int per,
                std::vector<BItem> &out) {
  for (const Seg &g : segs) {
    const int s0 = static_cast<int>(std::lower_bound(srow.begin(), srow.end(), g.r0) - srow.begin());
    const int s1 = static_cast<int>(std::lower_bound(srow.begin(), srow.end(), g.r1) - srow.begin());
    if (s0 >= static_cast<int>(srow.size()) || srow[s0] != g.r0 || s1 >= static_cast<int>(srow.size()) ||
        srow[s1] != g.r1)
      throw std::runtime_error("batched solver: work-list segment is not slice aligned");
    for (int a = s0; a < s1; a += per) out.push_back(BItem{g.sys, a, std::min(a + per, s1), g.c0});
  }
}

void row_items(const std::vector<Seg> &segs, int per, std::vector<BItem> &out) {
  for (const Seg &g : segs)
    for (int a = g.r0; a < g.r1; a += per) out.push_back(BItem{g.sys, a, std::min(a + per, g.r1), g.c0});
}

void items_for(const std::vector<Seg> &segs, int g, const std::vector<int> &srow, std::vector<BItem> &out) {
  if (g == 1) sell_items(segs, srow, kSellItemSlices, out);
  else row_items(segs, (256 / g) * kCsrvTrips, out);
}

// Block-diagonal concatenation: part i occupies rows [roff[i], ...) and its
// columns are shifted by coff[i].
Csr block_diag(const std::vector<const Csr *> &parts, const std::vector<int> &roff,
               const std::vector<int> &coff, int rows, int cols) {
  Csr m;
  m.rows = rows;
  m.cols = cols;
  m.rp.assign(rows + 1, 0);
  long long nnz = 0;
  for (size_t i = 0; i < parts.size(); ++i) {
    const Csr &p = *parts[i];
    for (int r = 0; r < p.rows; ++r) m.rp[roff[i] + r + 1] = p.rp[r + 1] - p.rp[r];
    nnz += p.nnz();
  }
  if (nnz > (1LL << 31) - (1LL << 26)) throw std::runtime_error("batched solver: too many nonzeros on one level");
  for (int r = 0; r < rows; ++r) m.rp[r + 1] += m.rp[r];
  m.ci.resize(nnz);
  m.v.resize(nnz);
  for (size_t i = 0; i < parts.size(); ++i) {
    const Csr &p = *parts[i];
    for (int r = 0; r < p.rows; ++r) {
      int d = m.rp[roff[i] + r];
      for (int e = p.rp[r]; e < p.rp[r + 1]; ++e, ++d) {
        m.ci[d] = p.ci[e] + coff[i];
        m.v[d] = p.v[e];
      }
    }
  }
  return m;
}

// ---------------------------------------------------------------------------
template <typename VT, int R>
class Batch final : public BatchSolver {
  using RV = Rv<VT, R>;
  using RD = Rv<double, R>;
  struct Range {
    int off = 0, count = 0;
  };
  struct BLevel {
    int n = 0;
    bool smoothed = false;
    DevSell<VT> A, P, Rs;
    DevCsrv<VT> C, Pc, Rc;
    int g = 1, pg = 1, rg = 1;
    RV *x = nullptr, *b = nullptr, *r = nullptr;
    std::vector<Range> fwd, bwd;
    Range whole_a, whole_p, below_r;
  };

 public:
  Batch(const std::vector<const Hierarchy *> &h, int nrhs, const SolverOptions &opt, int device);
  ~Batch() override;
  void solve_device(const double *b, double *x, cudaStream_t stream, std::vector<SolveStats> &st) override;
  void solve_host(const double *b, double *x, std::vector<SolveStats> &st) override;
  void set_tolerance(double tol, int max_iter) override {
    if (!(tol > 0.0)) throw std::runtime_error("CGSolver: tolerance must be positive.");
    if (max_iter < 0) throw std::runtime_error("CGSolver: maxIterations must be non-negative.");
    opt_.tol = tol;
    opt_.max_iter = max_iter;
  }
  int num_systems() const override { return S_; }
  int nrhs() const override { return nrhs_; }
  const std::vector<int> &system_rows() const override { return n_host_; }
  const std::vector<BatchLevelInfo> &level_info() const override { return info_; }
  long long launches() const override { return launches_; }
  double time_kernel(int kind, int reps, cudaStream_t stream) override;
  double time_level(int level, int op, int lanes, int reps, cudaStream_t stream) override;

 private:
  float time_level_op(int k, int op, int g, int reps);
  int grid(int count) const { return std::max(1, std::min(count, cap_blocks_)); }
  template <typename BT>
  void gs_pass(const BLevel &L, const BItem *it, int cnt, const Rv<BT, R> *b, RV *x, bool zero, cudaStream_t s);
  template <int kMode, typename BT>
  void spmv(const DevSell<VT> &Sm, const DevCsrv<VT> &Cm, int g, const BItem *it, int cnt, const RV *x, RV *y,
            const Rv<BT, R> *b, cudaStream_t s);
  template <typename BT>
  void smooth(int k, const Rv<BT, R> *b, RV *x, int steps, bool zero, cudaStream_t s);
  void vcycle(const RD *r0, RV *z, bool zero0, cudaStream_t s);
  void precondition(const RD *r, RV *z, cudaStream_t s) {
    for (int v = 0; v < opt_.vcycles; ++v) vcycle(r, z, v == 0, s);
  }
  void cg_start(cudaStream_t s);
  void cg_iteration(int parity, cudaStream_t s);
  void ensure_graphs();
  void run(std::vector<SolveStats> &st);
  void build_items();
  void autotune();
  float time_ms(const std::function<void()> &f, int reps);

  SolverOptions opt_;
  int device_ = 0, sms_ = 148, cap_blocks_ = 148 * 8;
  int S_ = 0, nrhs_ = 1, K_ = 0, n0_ = 0, maxn_ = 0;
  long long unknowns_ = 0;
  Layout ly_;
  Arena ar_;
  std::vector<BLevel> lv_;
  std::vector<BatchLevelInfo> info_;
  std::vector<int> n_host_;
  // work lists
  BItem *items_ = nullptr;
  size_t items_cap_ = 0;
  BItem *tmp_ = nullptr;  // work lists of timing runs
  size_t tmp_cap_ = 0;
  std::vector<BItem> h_items_;
  Range cg_range_, dense_range_;
  int *cg_first_ = nullptr;   // S + 1: first CG item of each system
  // coarsest levels
  double *ainv_ = nullptr;
  long long *ainv_off_ = nullptr;
  int *crow0_ = nullptr, *cn_ = nullptr;
  RV **xl_ = nullptr, **bl_ = nullptr;
  std::vector<BItem> dense_items_;
  // outer CG, FP64
  DevSell<double> cgA_;
  RD *x_ = nullptr, *r_ = nullptr, *p_ = nullptr, *ap_ = nullptr, *b_ = nullptr;
  RV *z_[2] = {nullptr, nullptr};
  double *partials_ = nullptr;
  BPair *pairs_ = nullptr;
  int *sys_done_ = nullptr;
  BCgShared *sh_ = nullptr, *host_sh_ = nullptr;
  double *ub_ = nullptr, *ux_ = nullptr;  // caller-layout staging of host solves
  // caller layout
  long long *uoff_ = nullptr, *qoff_ = nullptr;
  int *n_dev_ = nullptr, *off0_ = nullptr, *q0_ = nullptr;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraph_t graph_[2] = {nullptr, nullptr};
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
  long long launches_ = 0, graph_kernels_ = 0;
};

#define BKL(what) (cuda_check(cudaGetLastError(), what), ++launches_)

template <typename VT, int R>
Batch<VT, R>::Batch(const std::vector<const Hierarchy *> &h, int nrhs, const SolverOptions &opt, int device)
    : opt_(opt), device_(device) {
  if (h.empty()) throw std::runtime_error("batched solver: no systems");
  if (nrhs < 1 || nrhs > 4) throw std::runtime_error("batched solver: 1 to 4 right-hand sides per system");
  if (opt.smoother != 0 || opt.coarse_smoother > 0)
    throw std::runtime_error("batched solver: scalar multicolour Gauss-Seidel smoother only");
  if (opt.coarse != 1) throw std::runtime_error("batched solver: the coarsest level uses the dense solve (coarse_solver 1)");
  if (opt.reference_vcycle != 0) throw std::runtime_error("batched solver: reference_vcycle is not supported");
  if (!(opt.omega > 0.0 && opt.omega < 2.0)) throw std::runtime_error("smoother: omega must be in (0, 2).");
  if (opt.pre < 1 || opt.post < 1 || opt.vcycles < 1)
    throw std::runtime_error("Preconditioner requires at least one smoothing step.");
  if (opt.lanes != 0 && opt.lanes != 1 && opt.lanes != 2 && opt.lanes != 4 && opt.lanes != 8 && opt.lanes != 16 &&
      opt.lanes != 32)
    throw std::runtime_error("lanes must be 1, 2, 4, 8, 16 or 32");
  S_ = static_cast<int>(h.size());
  nrhs_ = nrhs;
  BCK(cudaSetDevice(device_));
  sms_ = sm_count(device_);
  cap_blocks_ = sms_ * 8;
  BCK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (auto &e : ev_) BCK(cudaEventCreate(&e));

  if (opt.coarse_rows < 0) throw std::runtime_error("coarse_rows must be >= 0");
  const std::vector<SysPrep> sp = prepare_all(h, true, opt.coarse_rows, opt.coloring);
  ly_ = make_layout(sp);
  K_ = ly_.K;
  n0_ = ly_.rows[0];
  lv_.resize(K_);
  info_.resize(K_);
  for (int s = 0; s < S_; ++s) {
    n_host_.push_back(sp[s].lv[0].A.rows);
    unknowns_ += n_host_.back();
    maxn_ = std::max(maxn_, n_host_.back());
  }

  // batch level matrices
  for (int k = 0; k < K_; ++k) {
    BLevel &L = lv_[k];
    L.n = ly_.rows[k];
    L.smoothed = !ly_.whole[k].empty();
    std::vector<const Csr *> parts;
    std::vector<int> off;
    for (int s = 0; s < S_; ++s)
      if (ly_.L[s] > k) parts.push_back(&sp[s].lv[k].A), off.push_back(ly_.off[k][s]);
    const Csr A = block_diag(parts, off, off, L.n, L.n);
    L.A = upload_sell(ar_, make_sell<VT>(A, ly_.bounds[k], true));
    L.C = upload_csrv<VT>(ar_, A, true);
    if (k == 0) cgA_ = upload_sell(ar_, make_sell<double>(A, ly_.bounds[0], true));
    info_[k].rows = L.n;
    info_[k].nnz = A.nnz();
    info_[k].systems = static_cast<int>(parts.size());
    info_[k].smoothed = static_cast<int>(ly_.whole[k].size());
    info_[k].max_colors = ly_.maxc[k];
    if (k + 1 < K_) {
      std::vector<const Csr *> pp, rr;
      std::vector<int> ro, co, rro, rco;
      for (int s = 0; s < S_; ++s) {
        if (ly_.L[s] - 1 <= k) continue;
        pp.push_back(&sp[s].lv[k].P), ro.push_back(ly_.off[k][s]), co.push_back(ly_.off[k + 1][s]);
        rr.push_back(&sp[s].lv[k].R), rro.push_back(ly_.off[k + 1][s]), rco.push_back(ly_.off[k][s]);
      }
      const Csr P = block_diag(pp, ro, co, L.n, ly_.rows[k + 1]);
      const Csr Rm = block_diag(rr, rro, rco, ly_.rows[k + 1], L.n);
      L.P = upload_sell(ar_, make_sell<VT>(P, ly_.sys_bounds[k], false));
      L.Rs = upload_sell(ar_, make_sell<VT>(Rm, ly_.sys_bounds[k + 1], false));
      L.Pc = upload_csrv<VT>(ar_, P, false);
      L.Rc = upload_csrv<VT>(ar_, Rm, false);
    }
    L.x = ar_.alloc<RV>(L.n);
    L.b = ar_.alloc<RV>(L.n);
    L.r = ar_.alloc<RV>(L.n);
    BCK(cudaMemset(L.x, 0, sizeof(RV) * L.n));
    BCK(cudaMemset(L.b, 0, sizeof(RV) * L.n));
    BCK(cudaMemset(L.r, 0, sizeof(RV) * L.n));
  }

  // coarsest levels: dense inverses and their work list
  {
    std::vector<long long> aoff(S_);
    std::vector<int> crow0(S_), cn(S_);
    long long tot = 0;
    for (int s = 0; s < S_; ++s) {
      const int lc = ly_.L[s] - 1, n = sp[s].lv[lc].A.rows;
      aoff[s] = tot;
      tot += static_cast<long long>(n) * n;
      crow0[s] = ly_.off[lc][s];
      cn[s] = n;
      for (int a = 0; a < n; a += kDenseItemRows) dense_items_.push_back(BItem{s, lc, a, std::min(a + kDenseItemRows, n)});
    }
    ainv_ = ar_.alloc<double>(tot);
    for (int s = 0; s < S_; ++s) {
      if (!sp[s].ainv.empty())
        BCK(cudaMemcpy(ainv_ + aoff[s], sp[s].ainv.data(), sizeof(double) * sp[s].ainv.size(), cudaMemcpyHostToDevice));
      else
        spd_inverse_device(sp[s].lv.back().A, ainv_ + aoff[s], stream_);
    }
    ainv_off_ = ar_.upload(aoff);
    crow0_ = ar_.upload(crow0);
    cn_ = ar_.upload(cn);
    std::vector<RV *> xs(K_), bs(K_);
    for (int k = 0; k < K_; ++k) xs[k] = lv_[k].x, bs[k] = lv_[k].b;
    xl_ = ar_.upload(xs);
    bl_ = ar_.upload(bs);
  }

  // outer CG vectors and state
  x_ = ar_.alloc<RD>(n0_);
  r_ = ar_.alloc<RD>(n0_);
  p_ = ar_.alloc<RD>(n0_);
  ap_ = ar_.alloc<RD>(n0_);
  b_ = ar_.alloc<RD>(n0_);
  z_[0] = ar_.alloc<RV>(n0_);
  z_[1] = ar_.alloc<RV>(n0_);
  for (void *p : {static_cast<void *>(x_), static_cast<void *>(r_), static_cast<void *>(p_),
                  static_cast<void *>(ap_), static_cast<void *>(b_)})
    BCK(cudaMemset(p, 0, sizeof(RD) * n0_));
  BCK(cudaMemset(z_[0], 0, sizeof(RV) * n0_));
  BCK(cudaMemset(z_[1], 0, sizeof(RV) * n0_));
  pairs_ = ar_.alloc<BPair>(static_cast<size_t>(S_) * R);
  BCK(cudaMemset(pairs_, 0, sizeof(BPair) * S_ * R));
  sys_done_ = ar_.alloc<int>(S_);
  BCK(cudaMemset(sys_done_, 0, sizeof(int) * S_));
  sh_ = ar_.alloc<BCgShared>(1);
  BCK(cudaMallocHost(&host_sh_, 2 * sizeof(BCgShared)));
  std::memset(host_sh_, 0, 2 * sizeof(BCgShared));
  ub_ = ar_.alloc<double>(static_cast<size_t>(unknowns_) * nrhs_);
  ux_ = ar_.alloc<double>(static_cast<size_t>(unknowns_) * nrhs_);

  // caller layout
  {
    std::vector<long long> uoff(S_), qoff(S_);
    std::vector<int> off0(S_), q0;
    long long u = 0;
    for (int s = 0; s < S_; ++s) {
      uoff[s] = u;
      u += static_cast<long long>(n_host_[s]) * nrhs_;
      qoff[s] = static_cast<long long>(q0.size());
      q0.insert(q0.end(), sp[s].q0.begin(), sp[s].q0.end());
      off0[s] = ly_.off[0][s];
    }
    uoff_ = ar_.upload(uoff);
    qoff_ = ar_.upload(qoff);
    off0_ = ar_.upload(off0);
    q0_ = ar_.upload(q0);
    n_dev_ = ar_.upload(n_host_);
  }

  // CG work list: level-0 slices of one system, kCgItemSlices per item
  {
    std::vector<int> first(S_ + 1, 0);
    std::vector<BItem> cgi;
    for (int s = 0; s < S_; ++s) {
      first[s] = static_cast<int>(cgi.size());
      const int o = ly_.off[0][s];
      sell_items({Seg{s, o, o + n_host_[s], o}}, cgA_.h_srow, kCgItemSlices, cgi);
    }
    first[S_] = static_cast<int>(cgi.size());
    cg_first_ = ar_.upload(first);
    partials_ = ar_.alloc<double>(3 * static_cast<size_t>(R) * std::max<size_t>(cgi.size(), 1));
    h_items_ = cgi;  // the CG list leads the item array (offset 0)
    cg_range_ = Range{0, static_cast<int>(cgi.size())};
  }

  if (opt_.lanes > 0) {
    for (BLevel &L : lv_) L.g = L.pg = L.rg = opt_.lanes;
  } else if (opt_.autotune) {
    autotune();
  }
  build_items();
  for (int k = 0; k < K_; ++k) {
    info_[k].lanes = lv_[k].g;
    info_[k].p_lanes = lv_[k].pg;
    info_[k].r_lanes = lv_[k].rg;
    long long it = 0;
    for (const Range &r : lv_[k].fwd) it += r.count;
    info_[k].sweep_items = it;
  }
}

template <typename VT, int R>
Batch<VT, R>::~Batch() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (int i = 0; i < 2; ++i) {
    if (exec_[i]) cudaGraphExecDestroy(exec_[i]);
    if (graph_[i]) cudaGraphDestroy(graph_[i]);
  }
  if (items_) cudaFree(items_);
  if (tmp_) cudaFree(tmp_);
  if (host_sh_) cudaFreeHost(host_sh_);
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  if (stream_) cudaStreamDestroy(stream_);
}

// Work lists of every pass for the current formats, after the CG list.
template <typename VT, int R>
void Batch<VT, R>::build_items() {
  std::vector<BItem> all(h_items_.begin(), h_items_.begin() + cg_range_.count);
  auto add = [&](const std::vector<Seg> &segs, int g, const std::vector<int> &srow) {
    Range r;
    r.off = static_cast<int>(all.size());
    items_for(segs, g, srow, all);
    r.count = static_cast<int>(all.size()) - r.off;
    return r;
  };
  for (int k = 0; k < K_; ++k) {
    BLevel &L = lv_[k];
    L.fwd.clear();
    L.bwd.clear();
    for (int j = 0; j < ly_.maxc[k]; ++j) {
      L.fwd.push_back(add(ly_.fwd[k][j], L.g, L.A.h_srow));
      L.bwd.push_back(add(ly_.bwd[k][j], L.g, L.A.h_srow));
    }
    L.whole_a = add(ly_.whole[k], L.g, L.A.h_srow);
    if (k + 1 < K_) {
      L.whole_p = add(ly_.whole[k], L.pg, L.P.h_srow);
      L.below_r = add(ly_.below[k], L.rg, L.Rs.h_srow);
    }
  }
  dense_range_.off = static_cast<int>(all.size());
  all.insert(all.end(), dense_items_.begin(), dense_items_.end());
  dense_range_.count = static_cast<int>(dense_items_.size());
  if (all.size() > items_cap_) {
    if (items_) BCK(cudaFree(items_));
    items_ = nullptr;
    BCK(cudaMalloc(&items_, sizeof(BItem) * all.size()));
    items_cap_ = all.size();
  }
  BCK(cudaMemcpy(items_, all.data(), sizeof(BItem) * all.size(), cudaMemcpyHostToDevice));
  h_items_ = all;
}

template <typename VT, int R>
template <typename BT>
void Batch<VT, R>::gs_pass(const BLevel &L, const BItem *it, int cnt, const Rv<BT, R> *b, RV *x, bool zero,
                           cudaStream_t s) {
  if (cnt <= 0) return;
  const VT w = VT(opt_.omega);
  const int gb = grid(cnt);
  if (L.g == 1) {
    if (zero) bsell_gs_kernel<VT, BT, R, true><<<gb, 256, 0, s>>>(L.A.view(), it, cnt, b, x, w, sys_done_);
    else bsell_gs_kernel<VT, BT, R, false><<<gb, 256, 0, s>>>(L.A.view(), it, cnt, b, x, w, sys_done_);
  } else {
    const CsrvView<VT> v = L.C.view();
#define BGS(G)                                                                                       \
  if (zero) bcsrv_gs_kernel<VT, BT, R, true, G><<<gb, 256, 0, s>>>(v, it, cnt, b, x, w, sys_done_);  \
  else bcsrv_gs_kernel<VT, BT, R, false, G><<<gb, 256, 0, s>>>(v, it, cnt, b, x, w, sys_done_);
    switch (L.g) {
      case 2: BGS(2) break;
      case 4: BGS(4) break;
      case 8: BGS(8) break;
      case 16: BGS(16) break;
      default: BGS(32) break;
    }
#undef BGS
  }
  BKL("batched gauss-seidel colour pass");
}

template <typename VT, int R>
template <int kMode, typename BT>
void Batch<VT, R>::spmv(const DevSell<VT> &Sm, const DevCsrv<VT> &Cm, int g, const BItem *it, int cnt,
                        const RV *x, RV *y, const Rv<BT, R> *b, cudaStream_t s) {
  if (cnt <= 0) return;
  const int gb = grid(cnt);
  if (g == 1) {
    bsell_spmv_kernel<VT, BT, R, kMode><<<gb, 256, 0, s>>>(Sm.view(), it, cnt, x, y, b, sys_done_);
  } else {
    const CsrvView<VT> v = Cm.view();
    switch (g) {
      case 2: bcsrv_spmv_kernel<VT, BT, R, kMode, 2><<<gb, 256, 0, s>>>(v, it, cnt, x, y, b, sys_done_); break;
      case 4: bcsrv_spmv_kernel<VT, BT, R, kMode, 4><<<gb, 256, 0, s>>>(v, it, cnt, x, y, b, sys_done_); break;
      case 8: bcsrv_spmv_kernel<VT, BT, R, kMode, 8><<<gb, 256, 0, s>>>(v, it, cnt, x, y, b, sys_done_); break;
      case 16: bcsrv_spmv_kernel<VT, BT, R, kMode, 16><<<gb, 256, 0, s>>>(v, it, cnt, x, y, b, sys_done_); break;
      default: bcsrv_spmv_kernel<VT, BT, R, kMode, 32><<<gb, 256, 0, s>>>(v, it, cnt, x, y, b, sys_done_); break;
    }
  }
  BKL("batched spmv");
}

// SymmetricGaussSeidelSmoother::smooth on every smoothed system of level k:
// forward pass j is colour j of each system, backward pass j its colour
// C_s - 1 - j.
template <typename VT, int R>
template <typename BT>
void Batch<VT, R>::smooth(int k, const Rv<BT, R> *b, RV *x, int steps, bool zero, cudaStream_t s) {
  const BLevel &L = lv_[k];
  for (int step = 0; step < steps; ++step) {
    for (const Range &r : L.fwd) gs_pass<BT>(L, items_ + r.off, r.count, b, x, zero && step == 0, s);
    for (const Range &r : L.bwd) gs_pass<BT>(L, items_ + r.off, r.count, b, x, false, s);
  }
}

template <typename VT, int R>
void Batch<VT, R>::vcycle(const RD *r0, RV *z, bool zero0, cudaStream_t s) {
  for (int k = 0; k + 1 < K_; ++k) {
    BLevel &L = lv_[k];
    if (k == 0) {
      smooth<double>(0, r0, z, opt_.pre, zero0, s);
      spmv<kSpmvResid, double>(L.A, L.C, L.g, items_ + L.whole_a.off, L.whole_a.count, z, L.r, r0, s);
    } else {
      smooth<VT>(k, L.b, L.x, opt_.pre, true, s);
      spmv<kSpmvResid, VT>(L.A, L.C, L.g, items_ + L.whole_a.off, L.whole_a.count, L.x, L.r, L.b, s);
    }
    spmv<kSpmvSet, VT>(L.Rs, L.Rc, L.rg, items_ + L.below_r.off, L.below_r.count, L.r, lv_[k + 1].b,
                       static_cast<const RV *>(nullptr), s);
  }
  bdense_kernel<VT, R><<<grid(dense_range_.count), 256, 0, s>>>(items_ + dense_range_.off, dense_range_.count,
                                                                 ainv_, ainv_off_, crow0_, cn_, xl_, bl_,
                                                                 sys_done_);
  BKL("batched coarsest solve");
  for (int k = K_ - 2; k >= 0; --k) {
    BLevel &L = lv_[k];
    RV *x = k == 0 ? z : L.x;
    spmv<kSpmvAdd, VT>(L.P, L.Pc, L.pg, items_ + L.whole_p.off, L.whole_p.count, lv_[k + 1].x, x,
                       static_cast<const RV *>(nullptr), s);
    if (k == 0) smooth<double>(0, r0, z, opt_.post, false, s);
    else smooth<VT>(k, L.b, L.x, opt_.post, false, s);
  }
}

template <typename VT, int R>
float Batch<VT, R>::time_ms(const std::function<void()> &f, int reps) {
  f();
  BCK(cudaEventRecord(ev_[2], stream_));
  for (int i = 0; i < reps; ++i) f();
  BCK(cudaEventRecord(ev_[3], stream_));
  BCK(cudaEventSynchronize(ev_[3]));
  float ms = 0.f;
  BCK(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
  return ms / reps;
}

// Threads per row for every level (one forward sweep over all systems) and
// transfer operator (one SpMV), chosen by timing each candidate on the
// solver's own buffers: SELL-32 with one lane per row, CSR-vector with
// 4/8/16/32 lanes.
// One operation of level k with g threads per row, on temporary work lists:
// op 0 a forward Gauss-Seidel sweep (all colour passes), 1 the residual,
// 2 the restriction to level k + 1, 3 the prolongation from it. Average ms.
template <typename VT, int R>
float Batch<VT, R>::time_level_op(int k, int op, int g, int reps) {
  BLevel &L = lv_[k];
  std::vector<BItem> v;
  std::vector<int> cnt;
  if (op == 0) {
    for (int j = 0; j < ly_.maxc[k]; ++j) {
      const size_t before = v.size();
      items_for(ly_.fwd[k][j], g, L.A.h_srow, v);
      cnt.push_back(static_cast<int>(v.size() - before));
    }
  } else if (op == 1) {
    items_for(ly_.whole[k], g, L.A.h_srow, v);
  } else if (op == 2) {
    items_for(ly_.below[k], g, L.Rs.h_srow, v);
  } else {
    items_for(ly_.whole[k], g, L.P.h_srow, v);
  }
  if (v.size() > tmp_cap_) {
    if (tmp_) BCK(cudaFree(tmp_));
    tmp_ = nullptr;
    BCK(cudaMalloc(&tmp_, sizeof(BItem) * v.size()));
    tmp_cap_ = v.size();
  }
  if (!v.empty()) BCK(cudaMemcpy(tmp_, v.data(), sizeof(BItem) * v.size(), cudaMemcpyHostToDevice));
  const int c = static_cast<int>(v.size());
  const int saved_g = L.g;
  L.g = g;
  const float ms = time_ms(
      [&] {
        if (op == 0) {
          int o = 0;
          for (int n : cnt) {
            if (k == 0) gs_pass<double>(L, tmp_ + o, n, r_, z_[0], false, stream_);
            else gs_pass<VT>(L, tmp_ + o, n, L.b, L.x, false, stream_);
            o += n;
          }
        } else if (op == 1) {
          if (k == 0) spmv<kSpmvResid, double>(L.A, L.C, g, tmp_, c, z_[0], L.r, r_, stream_);
          else spmv<kSpmvResid, VT>(L.A, L.C, g, tmp_, c, L.x, L.r, L.b, stream_);
        } else if (op == 2) {
          spmv<kSpmvSet, VT>(L.Rs, L.Rc, g, tmp_, c, L.r, lv_[k + 1].b, static_cast<const RV *>(nullptr), stream_);
        } else {
          spmv<kSpmvAdd, VT>(L.P, L.Pc, g, tmp_, c, lv_[k + 1].x, L.x, static_cast<const RV *>(nullptr), stream_);
        }
      },
      reps);
  L.g = saved_g;
  return ms;
}

template <typename VT, int R>
double Batch<VT, R>::time_level(int level, int op, int lanes, int reps, cudaStream_t stream) {
  if (level < 0 || level + 1 >= K_) throw std::runtime_error("time_level: level must have a coarser level below it");
  if (op < 0 || op > 3) throw std::runtime_error("time_level: op must be 0, 1, 2 or 3");
  if (lanes != 0 && lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    throw std::runtime_error("time_level: lanes must be 0, 1, 2, 4, 8, 16 or 32");
  const BLevel &L = lv_[level];
  const int g = lanes != 0 ? lanes : (op <= 1 ? L.g : op == 2 ? L.rg : L.pg);
  BCK(cudaSetDevice(device_));
  BCK(cudaEventRecord(ev_[0], stream));
  BCK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  BCK(cudaMemsetAsync(sys_done_, 0, sizeof(int) * S_, stream_));
  const long long saved = launches_;
  const float ms = time_level_op(level, op, g, std::max(1, reps));
  launches_ = saved;
  BCK(cudaEventRecord(ev_[1], stream_));
  BCK(cudaStreamWaitEvent(stream, ev_[1], 0));
  return ms;
}

// Threads per row for every level (one forward sweep over all systems) and
// transfer operator (one SpMV), chosen by timing each candidate on the
// solver's own buffers: SELL-32 with one lane per row, CSR-vector with
// 4/8/16/32 lanes.
template <typename VT, int R>
void Batch<VT, R>::autotune() {
  static const int cand[] = {1, 2, 4, 8, 16, 32};
  const long long saved = launches_;
  for (int k = 0; k + 1 < K_; ++k) {
    BLevel &L = lv_[k];
    int *choice[3] = {&L.g, &L.rg, &L.pg};
    const int ops[3] = {0, 2, 3};
    for (int w = 0; w < 3; ++w) {
      float best = 1e30f;
      int bg = 1;
      for (int g : cand) {
        const float ms = time_level_op(k, ops[w], g, 3);
        if (ms < best) best = ms, bg = g;
      }
      *choice[w] = bg;
    }
  }
  BCK(cudaStreamSynchronize(stream_));
  launches_ = saved;
  // the timing runs left values in the level buffers; clear them
  for (BLevel &L : lv_) {
    BCK(cudaMemset(L.x, 0, sizeof(RV) * L.n));
    BCK(cudaMemset(L.b, 0, sizeof(RV) * L.n));
    BCK(cudaMemset(L.r, 0, sizeof(RV) * L.n));
  }
  BCK(cudaMemset(z_[0], 0, sizeof(RV) * n0_));
}

template <typename VT, int R>
void Batch<VT, R>::cg_iteration(int parity, cudaStream_t s) {
  RV *z_old = z_[parity], *z_new = z_[parity ^ 1];
  const BItem *ci = items_ + cg_range_.off;
  const int nc = cg_range_.count, gb = grid(nc);
  bcg_spmv_pap_kernel<R><<<gb, 256, 0, s>>>(cgA_.view(), ci, nc, p_, ap_, sys_done_, partials_);
  BKL("batched cg spmv");
  bcg_finalize_kernel<R, kBFinPap><<<S_, 32 * R, 0, s>>>(cg_first_, partials_, pairs_, sys_done_, sh_);
  BKL("batched cg alpha");
  bcg_update_xr_kernel<R><<<gb, 256, 0, s>>>(cgA_.srow, ci, nc, x_, r_, p_, ap_, pairs_, sys_done_, partials_);
  BKL("batched cg update");
  bcg_finalize_kernel<R, kBFinXr><<<S_, 32 * R, 0, s>>>(cg_first_, partials_, pairs_, sys_done_, sh_);
  BKL("batched cg convergence");
  precondition(r_, z_new, s);
  bcg_dot_rz_kernel<VT, R><<<gb, 256, 0, s>>>(cgA_.srow, ci, nc, r_, z_new, opt_.flexible ? z_old : nullptr,
                                              sys_done_, partials_);
  BKL("batched cg dot");
  bcg_finalize_kernel<R, kBFinRz><<<S_, 32 * R, 0, s>>>(cg_first_, partials_, pairs_, sys_done_, sh_);
  BKL("batched cg beta");
  bcg_update_p_kernel<VT, R><<<gb, 256, 0, s>>>(cgA_.srow, ci, nc, z_new, p_, pairs_, sys_done_);
  BKL("batched cg p update");
}

// r = b - A x; z = M r; p = z; bb, rho, rr per pair.
template <typename VT, int R>
void Batch<VT, R>::cg_start(cudaStream_t s) {
  BCgShared init{};
  init.tol2 = opt_.tol * opt_.tol;
  init.max_iter = opt_.max_iter;
  init.flexible = opt_.flexible;
  init.active = 0;
  // pageable source: staged by the runtime before the call returns
  BCK(cudaMemcpyAsync(sh_, &init, sizeof(BCgShared), cudaMemcpyHostToDevice, s));
  BCK(cudaMemsetAsync(sys_done_, 0, sizeof(int) * S_, s));
  const BItem *ci = items_ + cg_range_.off;
  const int nc = cg_range_.count, gb = grid(nc);
  bsell_spmv_kernel<double, double, R, kSpmvResid><<<gb, 256, 0, s>>>(cgA_.view(), ci, nc, x_, r_, b_, nullptr);
  BKL("batched initial residual");
  precondition(r_, z_[0], s);
  bcg_init_kernel<VT, R><<<gb, 256, 0, s>>>(cgA_.srow, ci, nc, b_, r_, z_[0], p_, partials_);
  BKL("batched cg init");
  bcg_finalize_kernel<R, kBFinInit><<<S_, 32 * R, 0, s>>>(cg_first_, partials_, pairs_, sys_done_, sh_);
  BKL("batched cg init scalars");
}

template <typename VT, int R>
void Batch<VT, R>::ensure_graphs() {
  if (exec_[0] != nullptr) return;
  for (int par = 0; par < 2; ++par) {
    const long long before = launches_;
    BCK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cg_iteration(par, stream_);
    BCK(cudaStreamEndCapture(stream_, &graph_[par]));
    BCK(cudaGraphInstantiate(&exec_[par], graph_[par], 0));
    graph_kernels_ = launches_ - before;
    launches_ = before;  // captured, not executed
  }
}

template <typename VT, int R>
void Batch<VT, R>::run(std::vector<SolveStats> &out) {
  BCK(cudaEventRecord(ev_[2], stream_));
  cg_start(stream_);
  BCK(cudaMemcpyAsync(&host_sh_[0], sh_, sizeof(BCgShared), cudaMemcpyDeviceToHost, stream_));
  BCK(cudaStreamSynchronize(stream_));
  if (host_sh_[0].active > 0) {
    if (opt_.graph) {
      ensure_graphs();
      // One iteration queued ahead of the host check; the kernels of an
      // iteration queued after every system finished skip all their items.
      for (int it = 0; it < opt_.max_iter; ++it) {
        BCK(cudaGraphLaunch(exec_[it & 1], stream_));
        launches_ += graph_kernels_;
        BCK(cudaMemcpyAsync(&host_sh_[it & 1], sh_, sizeof(BCgShared), cudaMemcpyDeviceToHost, stream_));
        BCK(cudaEventRecord(ev_[it & 1], stream_));
        if (it >= 1) {
          BCK(cudaEventSynchronize(ev_[(it - 1) & 1]));
          if (host_sh_[(it - 1) & 1].active == 0) break;
        }
      }
    } else {
      for (int it = 0; it < opt_.max_iter; ++it) {
        cg_iteration(it & 1, stream_);
        BCK(cudaMemcpyAsync(&host_sh_[0], sh_, sizeof(BCgShared), cudaMemcpyDeviceToHost, stream_));
        BCK(cudaStreamSynchronize(stream_));
        if (host_sh_[0].active == 0) break;
      }
    }
  }
  BCK(cudaEventRecord(ev_[3], stream_));
  BCK(cudaEventSynchronize(ev_[3]));
  float ms = 0.f;
  BCK(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
  std::vector<BPair> hp(static_cast<size_t>(S_) * R);
  BCK(cudaMemcpy(hp.data(), pairs_, sizeof(BPair) * hp.size(), cudaMemcpyDeviceToHost));
  out.assign(static_cast<size_t>(S_) * nrhs_, SolveStats{});
  for (int s = 0; s < S_; ++s)
    for (int j = 0; j < nrhs_; ++j) {
      const BPair &p = hp[static_cast<size_t>(s) * R + j];
      SolveStats &o = out[static_cast<size_t>(s) * nrhs_ + j];
      o.iterations = p.iterations;
      o.status = p.status;
      o.ratio = p.ratio;
      o.bb = p.bb;
      o.spmv = p.iter;
      o.solve_ms = ms;
    }
}

template <typename VT, int R>
void Batch<VT, R>::solve_device(const double *b, double *x, cudaStream_t stream, std::vector<SolveStats> &st) {
  BCK(cudaSetDevice(device_));
  BCK(cudaEventRecord(ev_[0], stream));
  BCK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  const dim3 g(std::max(1, std::min(256, (maxn_ + 255) / 256)), S_);
  bscatter_kernel<R><<<g, 256, 0, stream_>>>(uoff_, n_dev_, off0_, qoff_, q0_, nrhs_, b, b_);
  bscatter_kernel<R><<<g, 256, 0, stream_>>>(uoff_, n_dev_, off0_, qoff_, q0_, nrhs_, x, x_);
  BKL("batched permute in");
  ++launches_;
  run(st);
  bgather_kernel<R><<<g, 256, 0, stream_>>>(uoff_, n_dev_, off0_, qoff_, q0_, nrhs_, x_, pairs_, x);
  BKL("batched permute out");
  BCK(cudaEventRecord(ev_[1], stream_));
  BCK(cudaStreamWaitEvent(stream, ev_[1], 0));
  BCK(cudaStreamSynchronize(stream));
}

template <typename VT, int R>
void Batch<VT, R>::solve_host(const double *b, double *x, std::vector<SolveStats> &st) {
  BCK(cudaSetDevice(device_));
  const size_t bytes = sizeof(double) * static_cast<size_t>(unknowns_) * nrhs_;
  BCK(cudaMemcpyAsync(ub_, b, bytes, cudaMemcpyHostToDevice, stream_));
  BCK(cudaMemcpyAsync(ux_, x, bytes, cudaMemcpyHostToDevice, stream_));
  solve_device(ub_, ux_, stream_, st);
  BCK(cudaMemcpyAsync(x, ux_, bytes, cudaMemcpyDeviceToHost, stream_));
  BCK(cudaStreamSynchronize(stream_));
}

template <typename VT, int R>
double Batch<VT, R>::time_kernel(int kind, int reps, cudaStream_t stream) {
  if (kind < 0 || kind > 2) throw std::runtime_error("time_kernel: kind must be 0, 1 or 2");
  if (reps < 1) reps = 1;
  BCK(cudaSetDevice(device_));
  BCK(cudaEventRecord(ev_[0], stream));
  BCK(cudaStreamWaitEvent(stream_, ev_[0], 0));
  BCK(cudaMemsetAsync(sys_done_, 0, sizeof(int) * S_, stream_));
  const BItem *ci = items_ + cg_range_.off;
  const int nc = cg_range_.count;
  const BLevel &L0 = lv_[0];
  std::function<void()> f;
  if (kind == 0)
    f = [&] {
      bcg_spmv_pap_kernel<R><<<grid(nc), 256, 0, stream_>>>(cgA_.view(), ci, nc, p_, ap_, sys_done_, partials_);
      BKL("batched cg spmv");
    };
  else if (kind == 1)
    f = [&] {
      for (const Range &r : L0.fwd) gs_pass<double>(L0, items_ + r.off, r.count, r_, z_[0], false, stream_);
    };
  else
    f = [&] { precondition(r_, z_[0], stream_); };
  const long long saved = launches_;
  const float ms = time_ms(f, reps);
  launches_ = saved;
  BCK(cudaEventRecord(ev_[1], stream_));
  BCK(cudaStreamWaitEvent(stream, ev_[1], 0));
  return ms;
}

}  // namespace

std::unique_ptr<BatchSolver> make_batch_solver(const std::vector<const Hierarchy *> &h, int nrhs,
                                               const SolverOptions &opt, int device) {
  const bool one = nrhs == 1;
  if (opt.mixed) {
    if (one) return std::unique_ptr<BatchSolver>(new Batch<float, 1>(h, nrhs, opt, device));
    return std::unique_ptr<BatchSolver>(new Batch<float, 4>(h, nrhs, opt, device));
  }
  if (one) return std::unique_ptr<BatchSolver>(new Batch<double, 1>(h, nrhs, opt, device));
  return std::unique_ptr<BatchSolver>(new Batch<double, 4>(h, nrhs, opt, device));
}

BatchPlanStats check_batch_plan(const std::vector<const Hierarchy *> &h) {
  const std::vector<SysPrep> sp = prepare_all(h, false, 0, 0);
  const Layout ly = make_layout(sp);
  BatchPlanStats st;
  st.levels = ly.K;
  auto fail = [](const std::string &m) { throw std::runtime_error("batch plan: " + m); };
  for (int k = 0; k < ly.K; ++k) {
    const std::vector<int> srow = slice_rows(ly.bounds[k], ly.rows[k]);
    // each smoothed system's rows: once in the forward passes, once in the backward passes
    for (int dir = 0; dir < 2; ++dir) {
      std::vector<int> seen(ly.rows[k], 0);
      const auto &passes = dir == 0 ? ly.fwd[k] : ly.bwd[k];
      for (size_t j = 0; j < passes.size(); ++j) {
        for (const Seg &g : passes[j]) {
          const int o = ly.off[k][g.sys];
          const int n = sp[g.sys].lv[k].A.rows, C = static_cast<int>(sp[g.sys].lv[k].cf.size()) - 1;
          const int c = dir == 0 ? static_cast<int>(j) : C - 1 - static_cast<int>(j);
          if (c < 0 || c >= C) fail("pass index outside the system's colours");
          if (g.r0 != o + sp[g.sys].lv[k].cf[c] || g.r1 != o + sp[g.sys].lv[k].cf[c + 1] || g.c0 != g.r0)
            fail("segment is not the system's colour range");
          if (g.r0 < o || g.r1 > o + n) fail("segment outside its system");
          for (int r = g.r0; r < g.r1; ++r) seen[r]++;
        }
        std::vector<BItem> v;
        sell_items(passes[j], srow, kSellItemSlices, v);
        std::vector<BItem> w;
        row_items(passes[j], 32, w);
        st.items += static_cast<long long>(v.size());
        // items cover exactly the segments, inside one system and one colour
        long long rows_items = 0, rows_segs = 0;
        for (const BItem &q : v) {
          const int o = ly.off[k][q.x], n = sp[q.x].lv[k].A.rows;
          if (srow[q.y] < o || srow[q.z] > o + n || q.z <= q.y) fail("SELL item crosses its system");
          if (srow[q.y] < q.w) fail("SELL item starts before its colour");
          rows_items += srow[q.z] - srow[q.y];
        }
        for (const BItem &q : w) {
          if (q.y < q.w || q.z <= q.y) fail("row item outside its colour");
        }
        for (const Seg &g : passes[j]) rows_segs += g.r1 - g.r0;
        if (rows_items != rows_segs) fail("SELL items do not cover the pass exactly");
      }
      for (int s = 0; s < ly.S; ++s) {
        if (ly.L[s] - 1 <= k) continue;
        const int o = ly.off[k][s], n = sp[s].lv[k].A.rows;
        for (int r = o; r < o + n; ++r)
          if (seen[r] != 1) fail("a row is not swept exactly once per direction");
      }
    }
    st.passes += 2 * static_cast<int>(ly.fwd[k].size());
  }
  return st;
}

}  // namespace gsb
