// The host setup (setup.cc) under AddressSanitizer and UndefinedBehaviorSanitizer:
// every routine the hierarchy build and the solver setup use -- SA hierarchy (both
// aggregations), HierarchicalReordering, both colourings, RCM, applyPermutation,
// permuteMatrix, HostELLMatrix, transpose, sparse products, node graph, block
// inverses -- on Poisson, GRF variable-coefficient, Kuhn P1 and 3x3 elasticity
// problems. Built and run by tests/test_sanitizers.py with 1 and 4 host threads.
#include "setup.h"
#include <cstdio>
#include <cstdlib>
#include <vector>
using namespace gsb;
static void exercise(const char *name, const Csr &a, int block) {
  for (int aggregation = 0; aggregation < 2; ++aggregation) {
    SaOptions o; o.block = block; o.eps_strong = 0.1; o.max_levels = 10; o.min_dofs = 20; o.aggregation = aggregation;
    Hierarchy h = build_hierarchy(a, o);
    std::vector<std::vector<int>> o2n, n2o;
    if (block == 1) hierarchical_reordering(h, o2n, n2o);
    for (size_t k = 0; k < h.A.size(); ++k) {
      const Csr &m = h.A[k];
      std::vector<int> c, v, off;
      greedy_coloring(m.rows, m.rp.data(), m.ci.data(), c, v, off);
      smallest_last_coloring(m.rows, m.rp.data(), m.ci.data(), c, v, off);
      std::vector<int> po(m.rows), pn(m.rows);
      rcm(m.rows, m.rp.data(), m.ci.data(), po.data(), pn.data());
      Csr ap = apply_permutation(m, po.data(), pn.data());
      Csr pm = permute_matrix(m, po.data(), po.data());
      HostEll e = build_ell(m, 5);
      Csr t = transpose(m);
      Csr s = spgemm(m, t);
      if (block == 3 && m.rows % 3 == 0) {
        std::vector<int> grp, gci; block_graph(m, 3, grp, gci);
        std::vector<double> d; block_inverses3x3(m, d);
      }
      (void)ap; (void)pm; (void)e; (void)s;
    }
    std::printf("%s aggregation %d: %zu levels\n", name, aggregation, h.A.size());
  }
}
int main() {
  exercise("poisson", poisson7(12, 11, 10), 1);
  exercise("grf", varcoef7(16, 16, 16, grf_coefficients(16, 16, 16, 8.0, 2.3, 4)), 1);
  exercise("kuhn", kuhn_laplacian(8, 0.2, 1), 1);
  std::vector<double> rhs;
  exercise("elasticity", elasticity_p1(6, 0.3, 2, rhs), 3);
  return 0;
}
