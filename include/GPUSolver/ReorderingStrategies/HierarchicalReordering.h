// gpuSolver::HierarchicalReordering (include/GPUSolver/ReorderingStrategies/
// HierarchicalReordering.h, src/ReorderingStrategies/HierarchicalReordering.cc:217-278
// of the reference): one permutation per level, finest first.
#pragma once
#include <vector>

#include "../detail/b200.h"

namespace gpuSolver {

struct HierarchicalReordering {
  std::vector<Permutation> compute(const AMGHierarchy &hierarchy) const {
    if (hierarchy.A.empty()) throw std::runtime_error("HierarchicalReordering: empty hierarchy.");
    if (hierarchy.R.size() + 1 != hierarchy.A.size())
      throw std::runtime_error("HierarchicalReordering: expected one restriction matrix between consecutive levels.");
    std::vector<gs_csr> A, P, R;
    for (const auto &m : hierarchy.A) A.push_back(m.view());
    for (const auto &m : hierarchy.P) P.push_back(m.view());
    for (const auto &m : hierarchy.R) R.push_back(m.view());
    gs_hierarchy *h = nullptr;
    detail::check(gs_hierarchy_from_levels(static_cast<int>(A.size()), A.data(), P.data(), R.data(), 1, &h));
    std::vector<std::vector<int>> o2n(A.size()), n2o(A.size());
    std::vector<int *> po, pn;
    for (size_t k = 0; k < A.size(); ++k) {
      o2n[k].resize(A[k].rows);
      n2o[k].resize(A[k].rows);
      po.push_back(o2n[k].data());
      pn.push_back(n2o[k].data());
    }
    const int rc = gs_hierarchical_reordering(h, po.data(), pn.data());
    gs_hierarchy_destroy(h);
    detail::check(rc);
    std::vector<Permutation> out;
    for (size_t k = 0; k < A.size(); ++k) out.emplace_back(o2n[k].size(), o2n[k].data(), n2o[k].data());
    return out;
  }
};

}  // namespace gpuSolver
