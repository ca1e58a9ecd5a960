// The oracle's restatement (oracle/oracle.cc) under AddressSanitizer and
// UndefinedBehaviorSanitizer: orc_amg_pcg on Poisson (SGS), Kuhn (damped Jacobi)
// and elasticity (3x3 block SGS, and the hybrid block GS / block Jacobi) with RCM
// permutations, FP64 / FP32 / mixed precision, smoother or dense coarsest level,
// with and without the reference's V-cycle aliasing and Polak-Ribiere CG, with
// half sweeps, and with strong-coupling colourings of the coarse levels.
// Built and run by tests/test_sanitizers.py; the oracle is the checker of the
// product, so its memory safety is checked as well.
#include "setup.h"
#include <cstdio>
#include <vector>
struct orc_csr { int rows, cols; const int *rowptr; const int *col; const double *val; };
struct orc_options { int smoother; int pre, post, coarse_steps, vcycles; double omega; int coarse_solver; int flexible;
  double tol; int max_iter; const double *colour_weights; const int *weight_offsets; int alias_correction; int coarse_smoother;
  const double *node_weights; const int *node_offsets; int half_sweeps;
  const int *colour_counts; const int *const *colour_verts; const int *const *colour_offs; int relaxed; };
extern "C" int orc_amg_pcg(int precision, int L, const orc_csr *A, const orc_csr *P, const orc_csr *R,
                           const int *const *o2n, const int *const *n2o, const orc_options *opt,
                           const double *b, double *x, int *iterations, int *status, double *ratio);
static orc_csr view(const gsb::Csr &m) { return orc_csr{m.rows, m.cols, m.rp.data(), m.ci.data(), m.v.data()}; }
static void run(const char *name, const gsb::Csr &a, int block, int smoother, int coarse_smoother) {
  gsb::SaOptions o; o.block = block; o.min_dofs = 30;
  gsb::Hierarchy h = gsb::build_hierarchy(a, o);
  std::vector<orc_csr> A, P, R;
  for (auto &m : h.A) A.push_back(view(m));
  for (auto &m : h.P) P.push_back(view(m));
  for (auto &m : h.R) R.push_back(view(m));
  std::vector<std::vector<int>> po, pn; std::vector<const int *> o2n, n2o;
  for (auto &m : h.A) { po.emplace_back(m.rows); pn.emplace_back(m.rows); gsb::rcm(m.rows, m.rp.data(), m.ci.data(), po.back().data(), pn.back().data()); }
  for (size_t k = 0; k < po.size(); ++k) o2n.push_back(po[k].data()), n2o.push_back(pn[k].data());
  std::vector<double> b = gsb::uniform_rhs(a.rows, 1);
  for (int precision = 0; precision < 3; ++precision)
    for (int coarse = 0; coarse < 2; ++coarse)
      for (int alias = 0; alias < 2; ++alias) {
        // half sweeps (forward pre-, backward post-smoothing) on the Gauss-Seidel
        // families with the dense coarsest level
        const int half = smoother <= 1 && coarse == 1 && alias == 0 ? 1 : 0;
        orc_options opt{smoother, 1, 1, 2, 1, smoother >= 2 ? 0.7 : 1.0, coarse, alias, 1e-8, 300, nullptr, nullptr, alias,
                        coarse_smoother, nullptr, nullptr, half, nullptr, nullptr, nullptr, 0};
        std::vector<double> x(a.rows, 0.0);
        int it = 0, st = 0; double ratio = 0;
        const int rc = orc_amg_pcg(precision, (int)A.size(), A.data(), P.data(), R.data(), o2n.data(), n2o.data(), &opt,
                                   b.data(), x.data(), &it, &st, &ratio);
        std::printf("%s p%d c%d a%d rc %d it %d st %d\n", name, precision, coarse, alias, rc, it, st);
      }
  // the strong-coupling colourings of the coarse Gauss-Seidel levels, computed
  // on each level as the oracle permutes it, with same-colour reads from the
  // sweep's starting iterate (FP64 and FP32, symmetric steps and half sweeps)
  if (smoother > 1 || coarse_smoother >= 0) return;
  const int L = static_cast<int>(A.size());
  std::vector<std::vector<int>> cv(L), co(L);
  std::vector<const int *> verts(L, nullptr), offs(L, nullptr);
  std::vector<int> counts(L, 0);
  for (int k = 1; k < L; ++k) {
    const gsb::Csr pk = gsb::permute_matrix(h.A[k], o2n[k], o2n[k]);
    std::vector<int> col;
    counts[k] = block == 3 ? gsb::relaxed_block_coloring(pk, 0.05, 0.5, col, cv[k], co[k])
                           : gsb::relaxed_coloring(pk.rows, pk.rp.data(), pk.ci.data(), pk.v.data(), 0.05, 0.5, col,
                                                   cv[k], co[k]);
    verts[k] = cv[k].data();
    offs[k] = co[k].data();
  }
  for (int precision = 0; precision < 2; ++precision)
    for (int half = 0; half < 2; ++half) {
      orc_options opt{smoother, 1, 1, 2, 1, 1.0, 1, 0, 1e-8, 300, nullptr, nullptr, 0, coarse_smoother, nullptr, nullptr,
                      half, counts.data(), verts.data(), offs.data(), 1};
      std::vector<double> x(a.rows, 0.0);
      int it = 0, st = 0; double ratio = 0;
      const int rc = orc_amg_pcg(precision, L, A.data(), P.data(), R.data(), o2n.data(), n2o.data(), &opt, b.data(),
                                 x.data(), &it, &st, &ratio);
      std::printf("%s-relaxed p%d h%d rc %d it %d st %d\n", name, precision, half, rc, it, st);
    }
}
int main() {
  run("poisson", gsb::poisson7(10, 9, 8), 1, 0, -1);
  run("kuhn-jacobi", gsb::kuhn_laplacian(7, 0.2, 1), 1, 2, -1);
  std::vector<double> rhs;
  gsb::Csr e = gsb::elasticity_p1(5, 0.3, 2, rhs);
  run("elasticity-bgs", e, 3, 1, -1);
  run("elasticity-hybrid", e, 3, 1, 3);
  return 0;
}
