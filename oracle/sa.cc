// ORACLE -- test infrastructure only. Only tests/ and bench.py's reference
// arm may load this code (as part of oracle/liboracle.so); the product never
// calls it.
//
// A C++ restatement of the smoothed-aggregation coarsening that the
// reference delegates to amgcl (examples/amgSolver/src/
// SmoothedAggregationCoarsener.cc:64-108; amgcl itself is absent and
// unpinned, cmake/recipes/amgcl.cmake:11-12), following the published
// method (Vanek, Mandel & Brezina, Computing 56, 1996) with the parameter
// choices of the numpy restatement in oracle/oracle.py (sa_coarsen,
// _sequential_aggregates, _sa_transfer, build_hierarchy), statement for
// statement and in the same summation order:
//   * node couplings: Frobenius norms of the block x block blocks;
//   * strength: w_ij^2 >= (eps^2 d_i) d_j, eps halved per level;
//   * aggregation: the three sequential steps in natural node order;
//   * tentative prolongator: one column per (aggregate, component),
//     1 / sqrt(aggregate size);
//   * filtered matrix: same-node and strong entries kept, the rest lumped
//     into the diagonal; omega = (4/3) / rho, rho the Gershgorin bound of
//     D_F^-1 A_F;
//   * P = (I - omega D_F^-1 A_F) P_tent, R = P^T, A_c = R (A P).
// The hierarchy loop is AMGHierarchyBuilder::build
// (examples/amgSolver/src/AMGHierarchyBuilder.cc:59-150): stop at
// <= min_dofs rows, at max_levels, or when a level does not shrink.
// It exists so that the reference arm of the benchmark can build its
// hierarchy without the product library, and so the numpy restatement has a
// fast twin at full sizes (tests/test_oracle_sa.py checks the two against
// each other and against the product's host build).
#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

thread_local std::string g_sa_err;

struct Mat {
  int rows = 0, cols = 0;
  std::vector<int> rp, ci;
  std::vector<double> v;
};

// C = A B, row by row: for each entry a_ik of row i in stored order, each
// entry b_kj of row k in stored order adds a_ik * b_kj to c_ij (the order
// scipy's csr_matmat sums in); columns sorted on output.
Mat multiply(const Mat &a, const Mat &b) {
  Mat c;
  c.rows = a.rows;
  c.cols = b.cols;
  c.rp.assign(a.rows + 1, 0);
  std::vector<double> acc(b.cols, 0.0);
  std::vector<int> mark(b.cols, -1), cols;
  for (int i = 0; i < a.rows; ++i) {
    cols.clear();
    for (int e = a.rp[i]; e < a.rp[i + 1]; ++e) {
      const int k = a.ci[e];
      const double av = a.v[e];
      for (int f = b.rp[k]; f < b.rp[k + 1]; ++f) {
        const int j = b.ci[f];
        if (mark[j] != i) {
          mark[j] = i;
          acc[j] = 0.0;
          cols.push_back(j);
        }
        acc[j] += av * b.v[f];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int j : cols) c.ci.push_back(j), c.v.push_back(acc[j]);
    c.rp[i + 1] = static_cast<int>(c.ci.size());
  }
  return c;
}

Mat transpose(const Mat &a) {
  Mat t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.rp.assign(a.cols + 1, 0);
  for (int j : a.ci) ++t.rp[j + 1];
  for (int j = 0; j < a.cols; ++j) t.rp[j + 1] += t.rp[j];
  t.ci.resize(a.ci.size());
  t.v.resize(a.v.size());
  std::vector<int> pos(t.rp.begin(), t.rp.end() - 1);
  for (int i = 0; i < a.rows; ++i)
    for (int e = a.rp[i]; e < a.rp[i + 1]; ++e) {
      const int p = pos[a.ci[e]]++;
      t.ci[p] = i;
      t.v[p] = a.v[e];
    }
  return t;
}

struct Level {
  Mat A, P, R;
};

// One coarsening step (oracle.py: sa_coarsen with aggregation 0). Returns
// false when the level has no aggregate.
bool coarsen(const Mat &a, int block, double eps, Mat &P, Mat &R, Mat &Ac) {
  const int n = a.rows;
  const int nn = n / block;
  // node couplings, neighbours in ascending node order
  std::vector<int> nrp(nn + 1, 0), nbr;
  std::vector<double> w, d(nn, 0.0);
  std::vector<std::pair<int, double>> acc;
  for (int i = 0; i < nn; ++i) {
    acc.clear();
    double dsum = 0.0;
    for (int r = block * i; r < block * i + block; ++r)
      for (int k = a.rp[r]; k < a.rp[r + 1]; ++k) {
        const int j = a.ci[k] / block;
        const double sq = a.v[k] * a.v[k];
        if (j == i) {
          dsum += sq;
        } else {
          auto it = std::find_if(acc.begin(), acc.end(), [j](const std::pair<int, double> &p) { return p.first == j; });
          if (it == acc.end()) acc.emplace_back(j, sq);
          else it->second += sq;
        }
      }
    d[i] = std::sqrt(dsum);
    std::sort(acc.begin(), acc.end(), [](const std::pair<int, double> &x, const std::pair<int, double> &y) {
      return x.first < y.first;
    });
    for (const auto &p : acc) nbr.push_back(p.first), w.push_back(std::sqrt(p.second));
    nrp[i + 1] = static_cast<int>(nbr.size());
  }
  const double eps2 = eps * eps;
  std::vector<char> strong(nbr.size());
  for (int i = 0; i < nn; ++i)
    for (int q = nrp[i]; q < nrp[i + 1]; ++q) strong[q] = w[q] * w[q] >= eps2 * d[i] * d[nbr[q]];

  // the three sequential aggregation steps
  std::vector<long long> agg(nn, -1);
  for (int i = 0; i < nn; ++i) {
    bool any = false;
    for (int q = nrp[i]; q < nrp[i + 1]; ++q) any = any || strong[q];
    if (!any) agg[i] = -2;  // isolated: no aggregate
  }
  long long nagg = 0;
  for (int i = 0; i < nn; ++i) {  // step 1: whole free strong neighbourhoods
    if (agg[i] != -1) continue;
    bool taken = false;
    for (int q = nrp[i]; q < nrp[i + 1]; ++q)
      if (strong[q] && agg[nbr[q]] != -1) taken = true;
    if (taken) continue;
    agg[i] = nagg;
    for (int q = nrp[i]; q < nrp[i + 1]; ++q)
      if (strong[q]) agg[nbr[q]] = nagg;
    ++nagg;
  }
  const std::vector<long long> agg1 = agg;
  for (int i = 0; i < nn; ++i) {  // step 2: join the strongest strongly coupled aggregate
    if (agg[i] != -1) continue;
    long long best = -1;
    double bw = -1.0;
    for (int q = nrp[i]; q < nrp[i + 1]; ++q)
      if (strong[q] && agg1[nbr[q]] >= 0 && w[q] > bw) bw = w[q], best = agg1[nbr[q]];
    if (best >= 0) agg[i] = best;
  }
  for (int i = 0; i < nn; ++i) {  // step 3: the rest start new aggregates
    if (agg[i] != -1) continue;
    agg[i] = nagg;
    for (int q = nrp[i]; q < nrp[i + 1]; ++q)
      if (strong[q] && agg[nbr[q]] == -1) agg[nbr[q]] = nagg;
    ++nagg;
  }
  if (nagg == 0) return false;

  // tentative prolongator
  std::vector<long long> size(nagg, 0);
  for (int i = 0; i < nn; ++i)
    if (agg[i] >= 0) ++size[agg[i]];
  const long long nc = nagg * block;
  std::vector<long long> tcol(n, -1);
  std::vector<double> tval(n, 0.0);
  for (int row = 0; row < n; ++row) {
    const int i = row / block, comp = row % block;
    if (agg[i] >= 0) {
      tcol[row] = agg[i] * block + comp;
      tval[row] = 1.0 / std::sqrt(static_cast<double>(size[agg[i]]));
    }
  }
  // filtered matrix: which entries are kept, and its diagonal
  std::vector<char> keep(a.ci.size(), 0);
  std::vector<double> fdiag(n, 0.0);
  for (int row = 0; row < n; ++row) {
    const int i = row / block;
    double dd = 0.0, lump = 0.0;
    for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
      const int j = a.ci[k] / block;
      bool kp = j == i;
      if (!kp)
        for (int q = nrp[i]; q < nrp[i + 1]; ++q)
          if (strong[q] && nbr[q] == j) {
            kp = true;
            break;
          }
      keep[k] = kp;
      if (a.ci[k] == row) dd += a.v[k];
      else if (!kp) lump += a.v[k];
    }
    fdiag[row] = dd + lump;
  }
  double rho = 0.0;
  for (int row = 0; row < n; ++row) {
    double s = std::fabs(fdiag[row]);
    for (int k = a.rp[row]; k < a.rp[row + 1]; ++k)
      if (keep[k] && a.ci[k] != row) s += std::fabs(a.v[k]);
    if (fdiag[row] != 0.0) rho = std::max(rho, s / std::fabs(fdiag[row]));
  }
  const double omega = rho > 0.0 ? (4.0 / 3.0) / rho : 0.0;
  // smoothed prolongator, coefficients summed per tentative column in the
  // order the row's entries are met
  P = Mat();
  P.rows = n;
  P.cols = static_cast<int>(nc);
  P.rp.assign(n + 1, 0);
  std::vector<std::pair<long long, double>> pacc;
  for (int row = 0; row < n; ++row) {
    const double scale = fdiag[row] != 0.0 ? omega / fdiag[row] : 0.0;
    pacc.clear();
    for (int k = a.rp[row]; k < a.rp[row + 1]; ++k) {
      if (!keep[k]) continue;
      const int c = a.ci[k];
      if (tcol[c] < 0) continue;
      const double afv = c == row ? fdiag[row] : a.v[k];
      const double coef = (c == row ? 1.0 : 0.0) - scale * afv;
      const long long t = tcol[c];
      auto it = std::find_if(pacc.begin(), pacc.end(), [t](const std::pair<long long, double> &p) { return p.first == t; });
      if (it == pacc.end()) pacc.emplace_back(t, coef * tval[c]);
      else it->second += coef * tval[c];
    }
    std::sort(pacc.begin(), pacc.end(), [](const std::pair<long long, double> &x, const std::pair<long long, double> &y) {
      return x.first < y.first;
    });
    for (const auto &p : pacc) P.ci.push_back(static_cast<int>(p.first)), P.v.push_back(p.second);
    P.rp[row + 1] = static_cast<int>(P.ci.size());
  }
  R = transpose(P);
  Ac = multiply(R, multiply(a, P));
  return true;
}

struct Hier {
  std::vector<Mat> A, P, R;
};

Mat from_raw(int rows, int cols, const int *rp, const int *ci, const double *v) {
  Mat m;
  m.rows = rows;
  m.cols = cols;
  m.rp.assign(rp, rp + rows + 1);
  m.ci.assign(ci, ci + rp[rows]);
  m.v.assign(v, v + rp[rows]);
  return m;
}

}  // namespace

extern "C" {

const char *orc_sa_last_error() { return g_sa_err.c_str(); }

// AMGHierarchyBuilder::build with the restated coarsener. *out owns the
// levels until orc_sa_free.
int orc_sa_build(int rows, const int *rp, const int *ci, const double *v, int block, double eps,
                 int max_levels, int min_dofs, void **out) {
  try {
    if (rows <= 0 || rp == nullptr || ci == nullptr || v == nullptr || out == nullptr || block < 1 ||
        rows % block != 0)
      throw std::runtime_error("orc_sa_build: bad arguments");
    std::unique_ptr<Hier> h(new Hier);
    h->A.push_back(from_raw(rows, rows, rp, ci, v));
    double e = eps;
    for (int level = 0; level < max_levels; ++level) {
      const Mat &cur = h->A.back();
      if (cur.rows <= min_dofs) break;
      Mat P, R, Ac;
      if (!coarsen(cur, block, e, P, R, Ac)) break;
      if (Ac.rows == 0 || Ac.rows >= cur.rows) break;
      h->P.push_back(std::move(P));
      h->R.push_back(std::move(R));
      h->A.push_back(std::move(Ac));
      e *= 0.5;
    }
    *out = h.release();
    return 0;
  } catch (const std::exception &ex) {
    g_sa_err = ex.what();
    return 1;
  }
}

int orc_sa_levels(const void *h) { return static_cast<int>(static_cast<const Hier *>(h)->A.size()); }

// which: 0 A_k, 1 P_k, 2 R_k. Sizes first (rp/ci/v null), then the arrays.
int orc_sa_matrix(const void *hv, int level, int which, int *rows, int *cols, int *nnz, int *rp, int *ci,
                  double *v) {
  const Hier *h = static_cast<const Hier *>(hv);
  const std::vector<Mat> &set = which == 0 ? h->A : (which == 1 ? h->P : h->R);
  if (level < 0 || level >= static_cast<int>(set.size())) {
    g_sa_err = "orc_sa_matrix: no such level";
    return 1;
  }
  const Mat &m = set[level];
  *rows = m.rows;
  *cols = m.cols;
  *nnz = static_cast<int>(m.ci.size());
  if (rp != nullptr) std::copy(m.rp.begin(), m.rp.end(), rp);
  if (ci != nullptr) std::copy(m.ci.begin(), m.ci.end(), ci);
  if (v != nullptr) std::copy(m.v.begin(), m.v.end(), v);
  return 0;
}

void orc_sa_free(void *h) { delete static_cast<Hier *>(h); }

}  // extern "C"
