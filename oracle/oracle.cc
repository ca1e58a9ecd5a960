// ORACLE -- test infrastructure only. Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg and reference arm may load this library,
// and only as the checker or the timed CPU baseline; the product never
// calls it.
//
// A plain CPU restatement of the reference's AMG-PCG path, templated on the
// precision of the outer CG (T) and of the V-cycle (V), so that
//   * T = V = float reproduces the reference's own FP32 arithmetic operation
//     for operation (pinned bit for bit against the reference compiled in
//     oracle/_ref, see tests/test_oracle_pin.py), and
//   * T = V = double is the FP64 oracle the GPU solver is compared with, and
//   * T = double, V = float checks the mixed-precision path.
// Each routine cites the reference code it restates. Sequential loops, CSR
// order summation, no FMA contraction (-ffp-contract=off), so results are
// reproducible.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

template <typename S>
struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> rp, ci;
  std::vector<S> v;
};

template <typename S>
Csr<S> from_raw(int rows, int cols, const int *rp, const int *ci, const double *v) {
  Csr<S> m;
  m.rows = rows;
  m.cols = cols;
  m.rp.assign(rp, rp + rows + 1);
  m.ci.assign(ci, ci + rp[rows]);
  m.v.resize(rp[rows]);
  for (int k = 0; k < rp[rows]; ++k) m.v[k] = static_cast<S>(v[k]);
  return m;
}

// permuteMatrix (src/SparseMatrixUtils.cc:8-31): (i, j) -> (ro2n[i], co2n[j]),
// columns sorted within each row (Eigen's setFromTriplets).
template <typename S>
Csr<S> permute_matrix(const Csr<S> &a, const int *ro2n, const int *co2n) {
  Csr<S> o;
  o.rows = a.rows;
  o.cols = a.cols;
  o.rp.assign(a.rows + 1, 0);
  for (int i = 0; i < a.rows; ++i) o.rp[ro2n[i] + 1] = a.rp[i + 1] - a.rp[i];
  for (int i = 0; i < a.rows; ++i) o.rp[i + 1] += o.rp[i];
  o.ci.resize(a.ci.size());
  o.v.resize(a.v.size());
  std::vector<std::pair<int, S>> row;
  for (int i = 0; i < a.rows; ++i) {
    row.clear();
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) row.push_back({co2n[a.ci[k]], a.v[k]});
    std::stable_sort(row.begin(), row.end(), [](const std::pair<int, S> &x, const std::pair<int, S> &y) {
      return x.first < y.first;
    });
    int d = o.rp[ro2n[i]];
    for (auto &e : row) o.ci[d] = e.first, o.v[d] = e.second, ++d;
  }
  return o;
}

// HostCSRMatrix::applyPermutation (src/HostSparseMatrix.cc:118-249).
template <typename S>
Csr<S> apply_permutation(const Csr<S> &a, const int *o2n, const int *n2o) {
  Csr<S> o;
  o.rows = o.cols = a.rows;
  o.rp.assign(a.rows + 1, 0);
  for (int i = 0; i < a.rows; ++i) o.rp[i + 1] = o.rp[i] + a.rp[n2o[i] + 1] - a.rp[n2o[i]];
  for (int i = 0; i < a.rows; ++i)
    for (int k = a.rp[n2o[i]]; k < a.rp[n2o[i] + 1]; ++k) {
      o.ci.push_back(o2n[a.ci[k]]);
      o.v.push_back(a.v[k]);
    }
  return o;
}

// GraphColoring::compute (src/GraphColoring.cc:9-72).
int coloring(int n, const int *rp, const int *ci, std::vector<int> &verts, std::vector<int> &offs) {
  std::vector<int> color(n, -1), forbid(n + 1, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j != i && color[j] >= 0) forbid[color[j]] = i;
    }
    int c = 0;
    while (forbid[c] == i) ++c;
    color[i] = c;
    nc = std::max(nc, c + 1);
  }
  offs.assign(nc + 1, 0);
  for (int i = 0; i < n; ++i) offs[color[i] + 1]++;
  for (int c = 0; c < nc; ++c) offs[c + 1] += offs[c];
  verts.assign(n, -1);
  std::vector<int> next(offs.begin(), offs.end() - 1);
  for (int i = 0; i < n; ++i) verts[next[color[i]]++] = i;
  return nc;
}

// buildBlockGraph (src/BlockUtils.cc:126-216).
template <typename S>
void block_graph(const Csr<S> &a, std::vector<int> &grp, std::vector<int> &gci) {
  const int nb = a.rows / 3;
  std::vector<std::vector<int>> adj(nb);
  for (int r = 0; r < a.rows; ++r)
    for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
      const int br = r / 3, bc = a.ci[k] / 3;
      if (br == bc) continue;
      adj[br].push_back(bc);
      adj[bc].push_back(br);
    }
  grp.assign(nb + 1, 0);
  gci.clear();
  for (int b = 0; b < nb; ++b) {
    std::sort(adj[b].begin(), adj[b].end());
    adj[b].erase(std::unique(adj[b].begin(), adj[b].end()), adj[b].end());
    grp[b + 1] = grp[b] + static_cast<int>(adj[b].size());
    gci.insert(gci.end(), adj[b].begin(), adj[b].end());
  }
}

// extractInverseDiagonalBlocks3x3 (src/BlockUtils.cc:218-277): Cholesky of
// each diagonal block, inverse by solving against the identity.
template <typename S>
std::vector<S> block_inverses(const Csr<S> &a) {
  const int nb = a.rows / 3;
  std::vector<S> inv(9 * static_cast<size_t>(nb));
  for (int b = 0; b < nb; ++b) {
    S m[3][3] = {};
    for (int lr = 0; lr < 3; ++lr)
      for (int k = a.rp[3 * b + lr]; k < a.rp[3 * b + lr + 1]; ++k) {
        const int c = a.ci[k] - 3 * b;
        if (c >= 0 && c < 3) m[lr][c] = a.v[k];
      }
    S l[3][3] = {};
    for (int j = 0; j < 3; ++j) {
      S d = m[j][j];
      for (int k = 0; k < j; ++k) d -= l[j][k] * l[j][k];
      if (!(d > S(0))) throw std::runtime_error("Block diagonal is not SPD.");
      l[j][j] = std::sqrt(d);
      for (int i = j + 1; i < 3; ++i) {
        S s = m[i][j];
        for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
        l[i][j] = s / l[j][j];
      }
    }
    for (int c = 0; c < 3; ++c) {
      S y[3];
      for (int i = 0; i < 3; ++i) {
        S s = (i == c) ? S(1) : S(0);
        for (int k = 0; k < i; ++k) s -= l[i][k] * y[k];
        y[i] = s / l[i][i];
      }
      for (int i = 2; i >= 0; --i) {
        S s = y[i];
        for (int k = i + 1; k < 3; ++k) s -= l[k][i] * y[k];
        y[i] = s / l[i][i];
      }
      for (int i = 0; i < 3; ++i) inv[9 * static_cast<size_t>(b) + 3 * i + c] = y[i];
    }
  }
  return inv;
}

// rowDotExcluding (src/CPU/CPUBackend.cc:62-86): sum over the row in CSR
// order, skipping columns in [ex_begin, ex_end); with `diag` non-null the
// diagonal entry is captured instead of summed.
template <typename S>
S row_dot(const Csr<S> &a, const S *x, int row, int ex_begin, int ex_end, S *diag) {
  S sum = S(0);
  if (diag) *diag = S(0);
  for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
    const int c = a.ci[k];
    if (c == row && diag) {
      *diag = a.v[k];
      continue;
    }
    if (c >= ex_begin && c < ex_end) continue;
    sum += a.v[k] * x[c];
  }
  return sum;
}

// CPUBackend::encodeSpmv (src/CPU/CPUBackend.cc:217-236).
template <typename S>
void spmv(const Csr<S> &a, const S *x, S *y) {
  for (int r = 0; r < a.rows; ++r) y[r] = row_dot(a, x, r, 0, 0, static_cast<S *>(nullptr));
}

// CPUBackend::encodeGaussSeidelColor (src/CPU/CPUBackend.cc:238-268).
template <typename S>
void gs_color(const Csr<S> &a, const int *order, int start, int count, const S *rhs, S *x, S w) {
  for (int k = start; k < start + count; ++k) {
    const int row = order[k];
    S d = S(0);
    const S off = row_dot(a, x, row, row, row + 1, &d);
    if (std::fabs(d) < S(1e-12)) throw std::runtime_error("zero diagonal entry.");
    const S nv = (rhs[row] - off) / d;
    x[row] = (S(1) - w) * x[row] + w * nv;
  }
}

// gs_color with the rows of colour `c` read from `xprev` (the iterate the
// sweep started with): Jacobi within the colour, Gauss-Seidel across colours.
template <typename S>
void gs_color_relaxed(const Csr<S> &a, const int *order, int start, int count, const S *rhs, S *x, const S *xprev,
                      const int *colour_of, int c, S w) {
  for (int k = start; k < start + count; ++k) {
    const int row = order[k];
    S d = S(0), off = S(0);
    for (int e = a.rp[row]; e < a.rp[row + 1]; ++e) {
      const int j = a.ci[e];
      if (j == row) d += a.v[e];
      else off += a.v[e] * (colour_of[j] == c ? xprev[j] : x[j]);
    }
    if (std::fabs(d) < S(1e-12)) throw std::runtime_error("zero diagonal entry.");
    const S nv = (rhs[row] - off) / d;
    x[row] = (S(1) - w) * x[row] + w * nv;
  }
}

// CPUBackend::encodeBlockGaussSeidelColor3x3 per-block formula
// (src/CPU/CPUBackend.cc:364-386), over colour entries [start, start+count)
// -- the (colorStart, colorCount) reading that BlockGaussSeidelSmoother
// passes (src/Smoothers/BlockGaussSeidelSmoother.cc:149-166).
template <typename S>
void block_gs_color(const Csr<S> &a, const int *order, int start, int count, const S *dinv,
                    const S *rhs, S *x, S w, const S *node_w = nullptr) {
  for (int k = start; k < start + count; ++k) {
    const int b = order[k], r0 = 3 * b;
    // a per-block scaling (no reference counterpart) replaces the colour's weight
    const S wb = node_w != nullptr ? node_w[b] : w;
    S res[3];
    for (int l = 0; l < 3; ++l) res[l] = rhs[r0 + l] - row_dot(a, x, r0 + l, r0, r0 + 3, static_cast<S *>(nullptr));
    const S *bi = dinv + 9 * static_cast<size_t>(b);
    for (int l = 0; l < 3; ++l) {
      S nv = S(0);
      for (int c = 0; c < 3; ++c) nv += bi[3 * l + c] * res[c];
      x[r0 + l] = (S(1) - wb) * x[r0 + l] + wb * nv;
    }
  }
}

// block_gs_color with the nodes of colour `c` read from `xprev` (the iterate
// the sweep started with): Jacobi within the colour, block Gauss-Seidel
// across colours. colour_of is per node.
template <typename S>
void block_gs_color_relaxed(const Csr<S> &a, const int *order, int start, int count, const S *dinv, const S *rhs,
                            S *x, const S *xprev, const int *colour_of, int c, S w, const S *node_w = nullptr) {
  for (int k = start; k < start + count; ++k) {
    const int b = order[k], r0 = 3 * b;
    const S wb = node_w != nullptr ? node_w[b] : w;
    S res[3];
    for (int l = 0; l < 3; ++l) {
      S off = S(0);
      for (int e = a.rp[r0 + l]; e < a.rp[r0 + l + 1]; ++e) {
        const int j = a.ci[e];
        if (j >= r0 && j < r0 + 3) continue;
        off += a.v[e] * (colour_of[j / 3] == c ? xprev[j] : x[j]);
      }
      res[l] = rhs[r0 + l] - off;
    }
    const S *bi = dinv + 9 * static_cast<size_t>(b);
    for (int l = 0; l < 3; ++l) {
      S nv = S(0);
      for (int q = 0; q < 3; ++q) nv += bi[3 * l + q] * res[q];
      x[r0 + l] = (S(1) - wb) * x[r0 + l] + wb * nv;
    }
  }
}

// CPUBackend::encodeDot (src/CPU/CPUBackend.cc:269-284), one thread.
template <typename S>
S dot(int n, const S *x, const S *y) {
  S s = S(0);
  for (int i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}

}  // namespace

// ---------------------------------------------------------------------------
// the multigrid preconditioner (MultigridSmoother) and CG (CGSolver)
// ---------------------------------------------------------------------------
extern "C" {

struct orc_csr {
  int rows, cols;
  const int *rowptr;
  const int *col;
  const double *val;
};

struct orc_options {
  int smoother;      // 0 multicolour SGS, 1 3x3 block SGS
  int pre, post, coarse_steps, vcycles;
  double omega;
  int coarse_solver; // 0 smoother steps, 1 dense Cholesky (FP64)
  int flexible;      // 0 beta = rho'/rho, 1 Polak-Ribiere
  double tol;
  int max_iter;
  const double *colour_weights;  // optional, per (level, colour), level-major
  const int *weight_offsets;     // levels + 1
  int alias_correction;          // 1: the reference's buffer aliasing at intermediate levels
  // smoother of the levels below the finest (MultigridSmoother's second type,
  // src/Smoothers/MultigridSmoother.cc:78-135); -1: the same as `smoother`.
  // Kinds: 0 SGS, 1 block SGS, 2 damped Jacobi, 3 block Jacobi, 4 identity.
  int coarse_smoother;
  // optional per-node weights of the block Gauss-Seidel levels, caller node
  // order, level after level (node_offsets: levels + 1, in nodes)
  const double *node_weights;
  const int *node_offsets;
  // 1: pre-smoothing is forward colour sweeps only and post-smoothing backward
  // only (the symmetric pair S, S^T of a textbook V-cycle); 0: symmetric
  // Gauss-Seidel steps, forward then backward, on both sides (the reference)
  int half_sweeps;
  // optional per-level colourings replacing the greedy one (a null level
  // keeps it): colour_counts[k] colours, colour_verts[k] the rows grouped by
  // colour, colour_offs[k] their offsets (counts + 1), rows of the level as
  // permuted by o2n. With `relaxed` 1 a colour pass on such a level reads the
  // rows of its own colour from the iterate its sweep started with (the
  // product's coloring 2, which lets weakly coupled rows share a colour).
  const int *colour_counts;
  const int *const *colour_verts;
  const int *const *colour_offs;
  int relaxed;
};

}  // extern "C"

namespace {

template <typename V>
struct Level {
  Csr<V> A;                 // permuteMatrix(A_k, pi_k, pi_k)
  Csr<V> P, R;              // to the next level (permuted)
  std::vector<int> verts, offs;
  int ncolors = 0;
  int kind = 0;             // smoother kind of this level (0 SGS, 1 BGS, 2 DJ, 3 BJ, 4 identity)
  std::vector<V> dinv;      // 3x3 block inverses (kinds 1, 3) or 1 / a_ii (kind 2)
  std::vector<V> rhs, x, res, corr, az;
  std::vector<double> chol; // coarsest Cholesky factor (row-major lower)
  std::vector<V> w;         // per-colour weights
  std::vector<V> nw;        // per-node weights (block levels), permuted node order, or empty
  bool relaxed = false;     // same-colour rows read from xprev (the sweep's starting iterate)
  std::vector<int> colour_of;
  std::vector<V> xprev;
};

template <typename T, typename V>
class Oracle {
 public:
  Oracle(int L, const orc_csr *A, const orc_csr *P, const orc_csr *R, const int *const *o2n,
         const int *const *n2o, const orc_options &o)
      : o_(o), lv_(L) {
    std::vector<std::vector<int>> id(L);
    auto perm = [&](int k) -> const int * {
      if (o2n != nullptr) return o2n[k];
      if (id[k].empty()) {
        id[k].resize(A[k].rows);
        for (int i = 0; i < A[k].rows; ++i) id[k][i] = i;
      }
      return id[k].data();
    };
    // MultigridSmoother constructor (src/Smoothers/MultigridSmoother.cc:197-335)
    for (int k = 0; k < L; ++k) {
      Level<V> &lv = lv_[k];
      const int *pk = perm(k);
      lv.A = permute_matrix(from_raw<V>(A[k].rows, A[k].cols, A[k].rowptr, A[k].col, A[k].val), pk, pk);
      const int n = lv.A.rows;
      lv.kind = (k > 0 && o.coarse_smoother >= 0) ? o.coarse_smoother : o.smoother;
      if (lv.kind == 1 || lv.kind == 3) {
        std::vector<int> grp, gci;
        block_graph(lv.A, grp, gci);
        lv.ncolors = coloring(n / 3, grp.data(), gci.data(), lv.verts, lv.offs);
        lv.dinv = block_inverses(lv.A);
        if (lv.kind == 1 && o.colour_verts != nullptr && o.colour_verts[k] != nullptr) {
          // a given node colouring (the product's) replaces the greedy one
          const int nn = n / 3;
          lv.ncolors = o.colour_counts[k];
          lv.verts.assign(o.colour_verts[k], o.colour_verts[k] + nn);
          lv.offs.assign(o.colour_offs[k], o.colour_offs[k] + lv.ncolors + 1);
          if (lv.offs.front() != 0 || lv.offs.back() != nn) throw std::runtime_error("colour offsets do not cover the level");
          lv.relaxed = o.relaxed != 0;
          lv.colour_of.assign(nn, -1);
          for (int c = 0; c < lv.ncolors; ++c)
            for (int q = lv.offs[c]; q < lv.offs[c + 1]; ++q) {
              const int node = lv.verts[q];
              if (node < 0 || node >= nn || lv.colour_of[node] >= 0) throw std::runtime_error("colour lists are not a partition");
              lv.colour_of[node] = c;
            }
          lv.xprev.assign(n, V(0));
        }
      } else {
        lv.ncolors = coloring(n, lv.A.rp.data(), lv.A.ci.data(), lv.verts, lv.offs);
        if (lv.kind == 0 && o.colour_verts != nullptr && o.colour_verts[k] != nullptr) {
          // a given colouring (the product's) replaces the greedy one
          lv.ncolors = o.colour_counts[k];
          lv.verts.assign(o.colour_verts[k], o.colour_verts[k] + n);
          lv.offs.assign(o.colour_offs[k], o.colour_offs[k] + lv.ncolors + 1);
          if (lv.offs.front() != 0 || lv.offs.back() != n) throw std::runtime_error("colour offsets do not cover the level");
          lv.relaxed = o.relaxed != 0;
          lv.colour_of.assign(n, -1);
          for (int c = 0; c < lv.ncolors; ++c)
            for (int q = lv.offs[c]; q < lv.offs[c + 1]; ++q) {
              const int row = lv.verts[q];
              if (row < 0 || row >= n || lv.colour_of[row] >= 0) throw std::runtime_error("colour lists are not a partition");
              lv.colour_of[row] = c;
            }
          lv.xprev.assign(n, V(0));
        }
        if (lv.kind == 2) {
          // DampedJacobiSmoother::initialize (src/Smoothers/DampedJacobiSmoother.cc:12-45)
          lv.dinv.assign(n, V(0));
          for (int i = 0; i < n; ++i) {
            bool found = false;
            for (int e = lv.A.rp[i]; e < lv.A.rp[i + 1]; ++e)
              if (lv.A.ci[e] == i) {
                if (std::fabs(double(lv.A.v[e])) < 1e-12)
                  throw std::runtime_error("DampedJacobiPreconditioner::initialize: zero diagonal entry.");
                lv.dinv[i] = V(1) / lv.A.v[e];
                found = true;
                break;
              }
            if (!found) throw std::runtime_error("DampedJacobiPreconditioner::initialize: missing diagonal entry.");
          }
        }
      }
      lv.rhs.assign(n, V(0));
      lv.x.assign(n, V(0));
      lv.res.assign(n, V(0));
      lv.corr.assign(n, V(0));
      lv.az.assign(n, V(0));
      lv.w.assign(lv.ncolors, V(o.omega));
      if (o.colour_weights != nullptr)
        for (int c = 0; c < lv.ncolors; ++c) lv.w[c] = V(o.colour_weights[o.weight_offsets[k] + c]);
      if (o.node_weights != nullptr && (lv.kind == 1 || lv.kind == 3)) {
        lv.nw.assign(n / 3, V(0));
        for (int i = 0; i < n / 3; ++i) lv.nw[pk[3 * i] / 3] = V(o.node_weights[o.node_offsets[k] + i]);
      }
      if (k > 0) {
        const int *pp = perm(k - 1);
        lv_[k - 1].P = permute_matrix(from_raw<V>(P[k - 1].rows, P[k - 1].cols, P[k - 1].rowptr, P[k - 1].col, P[k - 1].val), pp, pk);
        lv_[k - 1].R = permute_matrix(from_raw<V>(R[k - 1].rows, R[k - 1].cols, R[k - 1].rowptr, R[k - 1].col, R[k - 1].val), pk, pp);
      }
    }
    if (o.coarse_solver == 1) {
      // dense Cholesky of the coarsest permuted matrix, FP64
      Level<V> &c = lv_[L - 1];
      const int n = c.A.rows;
      const Csr<double> a64 = permute_matrix(from_raw<double>(A[L - 1].rows, A[L - 1].cols, A[L - 1].rowptr, A[L - 1].col, A[L - 1].val), perm(L - 1), perm(L - 1));
      c.chol.assign(static_cast<size_t>(n) * n, 0.0);
      std::vector<double> &m = c.chol;
      for (int i = 0; i < n; ++i)
        for (int k = a64.rp[i]; k < a64.rp[i + 1]; ++k) m[static_cast<size_t>(i) * n + a64.ci[k]] += a64.v[k];
      for (int j = 0; j < n; ++j) {
        double d = m[static_cast<size_t>(j) * n + j];
        for (int k = 0; k < j; ++k) d -= m[static_cast<size_t>(j) * n + k] * m[static_cast<size_t>(j) * n + k];
        if (!(d > 0.0)) throw std::runtime_error("coarsest level matrix is not SPD (Cholesky failed)");
        m[static_cast<size_t>(j) * n + j] = std::sqrt(d);
        for (int i = j + 1; i < n; ++i) {
          double s = m[static_cast<size_t>(i) * n + j];
          for (int k = 0; k < j; ++k) s -= m[static_cast<size_t>(i) * n + k] * m[static_cast<size_t>(j) * n + k];
          m[static_cast<size_t>(i) * n + j] = s / m[static_cast<size_t>(j) * n + j];
        }
      }
    }
    // CGSolver constructor: A' = applyPermutation(A_0, pi_0)
    // (src/CGSolver.cc:44-70, src/HostSparseMatrix.cc:57-63)
    cgA_ = apply_permutation(from_raw<T>(A[0].rows, A[0].cols, A[0].rowptr, A[0].col, A[0].val), perm(0), o2n ? n2o[0] : perm(0));
    n2o0_.assign(o2n ? n2o[0] : perm(0), (o2n ? n2o[0] : perm(0)) + A[0].rows);
  }

  // SymmetricGaussSeidelSmoother::smooth (src/Smoothers/SymmetricGaussSeidelSmoother.cc:80-128)
  // and BlockGaussSeidelSmoother::smooth (src/Smoothers/BlockGaussSeidelSmoother.cc:111-210).
  // dir: 0 forward + backward per step (the reference), 1 forward only,
  // 2 backward only (Gauss-Seidel kinds; the Jacobi kinds ignore it).
  void smooth(Level<V> &L, const V *rhs, V *x, int steps, int dir = 0) {
    if (L.kind == 4) {  // IdentityPreconditioner::apply: encodeCopy
      for (int i = 0; i < L.A.rows; ++i) x[i] = rhs[i];
      return;
    }
    if (steps == 0) throw std::runtime_error("Preconditioner requires at least one smoothing step.");
    if (L.kind == 2 || L.kind == 3) {
      // DampedJacobiSmoother::smooth (src/Smoothers/DampedJacobiSmoother.cc:55-67),
      // BlockJacobiSmoother::smooth (src/Smoothers/BlockJacobiSmoother.cc:33-69):
      // Az = A x; c = rhs; c += -1 Az; c <- D^-1 c; x += omega c
      const int n = L.A.rows;
      for (int s = 0; s < steps; ++s) {
        spmv(L.A, x, L.az.data());
        for (int i = 0; i < n; ++i) L.res[i] = rhs[i];
        for (int i = 0; i < n; ++i) L.res[i] += V(-1) * L.az[i];
        if (L.kind == 2) {
          for (int i = 0; i < n; ++i) L.corr[i] = L.res[i] * L.dinv[i];
        } else {
          for (int b = 0; b < n / 3; ++b)
            for (int r = 0; r < 3; ++r) {
              V sum = V(0);
              for (int c = 0; c < 3; ++c) sum += L.dinv[9 * b + 3 * r + c] * L.res[3 * b + c];
              L.corr[3 * b + r] = sum;
            }
        }
        for (int i = 0; i < n; ++i) x[i] += V(o_.omega) * L.corr[i];
      }
      return;
    }
    const int n = L.A.rows;
    for (int s = 0; s < steps; ++s) {
      if (dir != 2) {
        if (L.relaxed) std::copy(x, x + n, L.xprev.begin());
        for (int c = 0; c < L.ncolors; ++c) pass(L, c, rhs, x);
      }
      if (dir != 1) {
        if (L.relaxed) std::copy(x, x + n, L.xprev.begin());
        for (int c = L.ncolors; c > 0; --c) pass(L, c - 1, rhs, x);
      }
    }
  }
  void pass(Level<V> &L, int c, const V *rhs, V *x) {
    const int start = L.offs[c], count = L.offs[c + 1] - L.offs[c];
    if (L.kind == 1 && L.relaxed) {
      if (count == 0) return;
      block_gs_color_relaxed(L.A, L.verts.data(), start, count, L.dinv.data(), rhs, x, L.xprev.data(),
                             L.colour_of.data(), c, L.w[c], L.nw.empty() ? static_cast<const V *>(nullptr) : L.nw.data());
    } else if (L.kind == 1) {
      if (count == 0) return;
      block_gs_color(L.A, L.verts.data(), start, count, L.dinv.data(), rhs, x, L.w[c],
                     L.nw.empty() ? static_cast<const V *>(nullptr) : L.nw.data());
    } else if (L.relaxed) {
      gs_color_relaxed(L.A, L.verts.data(), start, count, rhs, x, L.xprev.data(), L.colour_of.data(), c, L.w[c]);
    } else {
      gs_color(L.A, L.verts.data(), start, count, rhs, x, L.w[c]);
    }
  }

  // MultigridSmoother::vCycle (src/Smoothers/MultigridSmoother.cc:337-412).
  void vcycle(int k, const V *rhs, V *x) {
    Level<V> &L = lv_[k];
    const int n = L.A.rows;
    if (k + 1 == static_cast<int>(lv_.size())) {
      if (o_.coarse_solver == 1) {
        std::vector<double> y(n);
        const std::vector<double> &m = L.chol;
        for (int i = 0; i < n; ++i) {
          double s = double(rhs[i]);
          for (int j = 0; j < i; ++j) s -= m[static_cast<size_t>(i) * n + j] * y[j];
          y[i] = s / m[static_cast<size_t>(i) * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
          double s = y[i];
          for (int j = i + 1; j < n; ++j) s -= m[static_cast<size_t>(j) * n + i] * y[j];
          y[i] = s / m[static_cast<size_t>(i) * n + i];
        }
        for (int i = 0; i < n; ++i) x[i] = V(y[i]);
      } else {
        smooth(L, rhs, x, o_.coarse_steps);
      }
      return;
    }
    smooth(L, rhs, x, o_.pre, o_.half_sweeps ? 1 : 0);
    spmv(L.A, x, L.az.data());
    for (int i = 0; i < n; ++i) L.res[i] = rhs[i];                 // encodeCopy
    for (int i = 0; i < n; ++i) L.res[i] += V(-1) * L.az[i];       // encodeAxpy(-1)
    Level<V> &C = lv_[k + 1];
    spmv(L.R, L.res.data(), C.rhs.data());
    std::fill(C.x.begin(), C.x.end(), V(0));                       // encodeSetZero
    vcycle(k + 1, C.rhs.data(), C.x.data());
    if (o_.alias_correction && k > 0) {
      // The reference recurses with vCycle(k+1, coarse.rhs, coarse.correction)
      // (src/Smoothers/MultigridSmoother.cc:394-395), so on every level below
      // the finest `solution` IS levels_[k].correction; the prolongation
      // (:401-402) then overwrites the solution and the axpy (:404) doubles
      // it: x_k = 2 P x_{k+1}, the pre-smoothed x_k is lost.
      spmv(L.P, C.x.data(), x);
      for (int i = 0; i < n; ++i) x[i] += V(1) * x[i];
    } else {
      spmv(L.P, C.x.data(), L.corr.data());
      for (int i = 0; i < n; ++i) x[i] += V(1) * L.corr[i];          // encodeAxpy(1)
    }
    smooth(L, rhs, x, o_.post, o_.half_sweeps ? 2 : 0);
  }

  // Multigrid*Preconditioner::apply: z = 0, then `vcycles` V-cycles.
  void apply(const std::vector<T> &r, std::vector<T> &z) {
    Level<V> &L = lv_[0];
    const int n = L.A.rows;
    std::vector<V> rv(n), zv(n, V(0));
    for (int i = 0; i < n; ++i) rv[i] = V(r[i]);
    for (int v = 0; v < o_.vcycles; ++v) vcycle(0, rv.data(), zv.data());
    for (int i = 0; i < n; ++i) z[i] = T(zv[i]);
  }

  // CGSolver::solve (src/CGSolver.cc:87-306). Returns the reference's
  // iteration count; *status: 1 converged, 2 max iterations, 5 converged
  // before the loop, 6 zero right-hand side.
  int solve(const T *b_in, T *x_in, int *status, double *ratio_out) {
    const int n = cgA_.rows;
    std::vector<T> b(n), x(n);
    for (int i = 0; i < n; ++i) b[i] = b_in[n2o0_[i]], x[i] = x_in[n2o0_[i]];
    double bn = 0.0;
    for (int i = 0; i < n; ++i) bn += double(b_in[i]) * double(b_in[i]);
    if (std::sqrt(bn) < 1e-12) {
      for (int i = 0; i < n; ++i) x_in[i] = T(0);
      *status = 6;
      return 0;
    }
    std::vector<T> ax(n), r(n), z(n), z1(n), p(n), ap(n), r1(n);
    spmv(cgA_, x.data(), ax.data());
    r = b;
    for (int i = 0; i < n; ++i) r[i] += T(-1) * ax[i];
    apply(r, z);
    p = z;
    const T bb = dot(n, b.data(), b.data());
    T rho = dot(n, r.data(), z.data());
    T rr = dot(n, r.data(), r.data());
    T ratio = rr / bb;
    const T tol = T(o_.tol);
    if (!std::isfinite(double(ratio))) throw std::runtime_error("CGSolver: initial residual is NaN/Inf");
    if (ratio < tol * tol) {
      *status = 5;
      *ratio_out = double(ratio);
      return 0;
    }
    int iters = 0;
    *status = 2;
    for (int itr = 0; itr < o_.max_iter; ++itr) {
      spmv(cgA_, p.data(), ap.data());
      const T pap = dot(n, p.data(), ap.data());
      const T alpha = rho / pap;
      for (int i = 0; i < n; ++i) x[i] += alpha * p[i];
      const T nalpha = -alpha;
      r1 = r;
      for (int i = 0; i < n; ++i) r1[i] += nalpha * ap[i];
      rr = dot(n, r1.data(), r1.data());
      ratio = rr / bb;
      apply(r1, z1);
      T rho1 = dot(n, r1.data(), z1.data());
      T beta;
      if (o_.flexible) {
        const T rzo = dot(n, r1.data(), z.data());
        beta = (rho1 - rzo) / rho;
      } else {
        beta = rho1 / rho;
      }
      for (int i = 0; i < n; ++i) p[i] *= beta;          // encodeScale
      for (int i = 0; i < n; ++i) p[i] += T(1) * z1[i];  // encodeAxpy(1)
      if (!std::isfinite(double(ratio))) throw std::runtime_error("CGSolver: solver diverged (NaN/Inf residual).");
      if (ratio < tol * tol) {
        iters = itr;
        *status = 1;
        break;
      }
      rho = rho1;  // swap(rhoDev, rhoNewDev)
      std::swap(r, r1);
      std::swap(z, z1);
      if (itr == o_.max_iter - 1) iters = o_.max_iter;
    }
    for (int i = 0; i < n; ++i) x_in[n2o0_[i]] = x[i];
    *ratio_out = double(ratio);
    return iters;
  }

 private:
  orc_options o_;
  std::vector<Level<V>> lv_;
  Csr<T> cgA_;
  std::vector<int> n2o0_;
};

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

// precision: 0 = FP64 throughout, 1 = FP32 throughout (the reference's
// arithmetic), 2 = FP64 CG with an FP32 V-cycle.
int orc_amg_pcg(int precision, int L, const orc_csr *A, const orc_csr *P, const orc_csr *R,
                const int *const *o2n, const int *const *n2o, const orc_options *opt,
                const double *b, double *x, int *iterations, int *status, double *ratio) {
  return guarded([&] {
    const int n = A[0].rows;
    if (precision == 1) {
      Oracle<float, float> orc(L, A, P, R, o2n, n2o, *opt);
      std::vector<float> bf(b, b + n), xf(x, x + n);
      *iterations = orc.solve(bf.data(), xf.data(), status, ratio);
      for (int i = 0; i < n; ++i) x[i] = xf[i];
    } else if (precision == 2) {
      Oracle<double, float> orc(L, A, P, R, o2n, n2o, *opt);
      std::vector<double> xv(x, x + n);
      *iterations = orc.solve(b, xv.data(), status, ratio);
      std::memcpy(x, xv.data(), sizeof(double) * n);
    } else {
      Oracle<double, double> orc(L, A, P, R, o2n, n2o, *opt);
      std::vector<double> xv(x, x + n);
      *iterations = orc.solve(b, xv.data(), status, ratio);
      std::memcpy(x, xv.data(), sizeof(double) * n);
    }
  });
}

// One preconditioner application z = M r (arrays in the level-0 order of the
// caller, i.e. permuted by permutation[0] as CGSolver does before applying).
int orc_precondition(int precision, int L, const orc_csr *A, const orc_csr *P, const orc_csr *R,
                     const int *const *o2n, const int *const *n2o, const orc_options *opt,
                     const double *r, double *z) {
  return guarded([&] {
    const int n = A[0].rows;
    if (precision == 1) {
      Oracle<float, float> orc(L, A, P, R, o2n, n2o, *opt);
      std::vector<float> rv(r, r + n), zv(n);
      orc.apply(rv, zv);
      for (int i = 0; i < n; ++i) z[i] = zv[i];
    } else {
      Oracle<double, double> orc(L, A, P, R, o2n, n2o, *opt);
      std::vector<double> rv(r, r + n), zv(n);
      orc.apply(rv, zv);
      std::memcpy(z, zv.data(), sizeof(double) * n);
    }
  });
}

// Kernel-level restatements in FP64 and FP32.
void orc_spmv_f64(int rows, int cols, const int *rp, const int *ci, const double *v,
                  const double *x, double *y) {
  spmv(from_raw<double>(rows, cols, rp, ci, v), x, y);
}
void orc_spmv_f32(int rows, int cols, const int *rp, const int *ci, const double *v,
                  const float *x, float *y) {
  spmv(from_raw<float>(rows, cols, rp, ci, v), x, y);
}
int orc_gs_color_f64(int n, const int *rp, const int *ci, const double *v, const int *order,
                     int start, int count, const double *rhs, double *x, double w) {
  return guarded([&] { gs_color(from_raw<double>(n, n, rp, ci, v), order, start, count, rhs, x, w); });
}
int orc_gs_color_f32(int n, const int *rp, const int *ci, const double *v, const int *order,
                     int start, int count, const float *rhs, float *x, float w) {
  return guarded([&] { gs_color(from_raw<float>(n, n, rp, ci, v), order, start, count, rhs, x, w); });
}
int orc_block_gs_color_f64(int n, const int *rp, const int *ci, const double *v, const int *order,
                           int start, int count, const double *dinv, const double *rhs, double *x,
                           double w) {
  return guarded([&] { block_gs_color(from_raw<double>(n, n, rp, ci, v), order, start, count, dinv, rhs, x, w); });
}
int orc_block_inverses_f64(int n, const int *rp, const int *ci, const double *v, double *dinv) {
  return guarded([&] {
    const std::vector<double> d = block_inverses(from_raw<double>(n, n, rp, ci, v));
    std::memcpy(dinv, d.data(), sizeof(double) * d.size());
  });
}
double orc_dot_f64(int n, const double *x, const double *y) { return dot(n, x, y); }
float orc_dot_f32(int n, const float *x, const float *y) { return dot(n, x, y); }
int orc_coloring(int n, const int *rp, const int *ci, int *verts, int *offs) {
  std::vector<int> v, o;
  const int nc = coloring(n, rp, ci, v, o);
  std::memcpy(verts, v.data(), sizeof(int) * n);
  std::memcpy(offs, o.data(), sizeof(int) * (nc + 1));
  return nc;
}

}  // extern "C"
