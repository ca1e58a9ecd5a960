// gpuSolver::SmoothedAggregationCoarsener + AMGHierarchyBuilder
// (examples/amgSolver/include/AMGUtils/*.h of the reference). The coarsener
// restates smoothed aggregation from the published method (Vanek, Mandel &
// Brezina 1996); the reference uses amgcl for it.
#pragma once
#include <cstddef>

#include "detail/b200.h"

namespace gpuSolver {

class SmoothedAggregationCoarsener {
 public:
  SmoothedAggregationCoarsener(int blockSize, float epsStrong) : blockSize_(blockSize), epsStrong_(epsStrong) {
    if (blockSize_ <= 0) throw std::runtime_error("block size must be positive.");
  }
  int blockSize() const { return blockSize_; }
  float epsStrong() const { return epsStrong_; }

 private:
  int blockSize_;
  float epsStrong_;
};

class AMGHierarchyBuilder {
 public:
  AMGHierarchyBuilder(const SmoothedAggregationCoarsener &coarsener, int maxLevels, int minDofs)
      : coarsener_(coarsener), maxLevels_(maxLevels), minDofs_(minDofs) {
    if (maxLevels_ <= 0) throw std::runtime_error("AMGHierarchyBuilder: maxLevels must be positive.");
    if (minDofs_ <= 0) throw std::runtime_error("AMGHierarchyBuilder: minDofs must be positive.");
  }
  AMGHierarchy build(const CsrMatrix &matrix) const { return run(matrix, false, 0); }
  // build(matrix, nearNullspace) (examples/amgSolver/src/AMGHierarchyBuilder.cc:59-150):
  // without near-nullspace modes it is build(matrix). Modes (the reference hands
  // them, orthonormalised, to amgcl's tentative prolongator) are not supported
  // here: a non-null argument throws instead of being ignored.
  AMGHierarchy build(const CsrMatrix &matrix, std::nullptr_t) const { return build(matrix); }
  template <typename Modes>
  AMGHierarchy build(const CsrMatrix &matrix, const Modes *nearNullspace) const {
    if (nearNullspace != nullptr)
      throw std::runtime_error("AMGHierarchyBuilder: near-nullspace modes are not supported by this library.");
    return build(matrix);
  }
  // Extension (no reference counterpart): the hierarchy built on GPU `device`
  // with the distance-2 independent-set aggregation (gs_hierarchy_build_ex);
  // rows of `matrix` need sorted, duplicate-free column indices.
  AMGHierarchy buildOnDevice(const CsrMatrix &matrix, int device = 0) const { return run(matrix, true, device); }

 private:
  AMGHierarchy run(const CsrMatrix &matrix, bool on_device, int device) const {
    gs_host_csr *m = nullptr;
    detail::check(gs_host_csr_create(matrix.rows(), matrix.cols(), matrix.rowPtr.data(),
                                     matrix.colIdx.data(), matrix.values.data(), &m));
    gs_hierarchy *h = nullptr;
    const int rc = on_device ? gs_hierarchy_build_ex(m, coarsener_.blockSize(), coarsener_.epsStrong(), maxLevels_,
                                                     minDofs_, 1, device, nullptr, &h)
                             : gs_hierarchy_build(m, coarsener_.blockSize(), coarsener_.epsStrong(), maxLevels_,
                                                  minDofs_, &h);
    gs_host_csr_destroy(m);
    detail::check(rc);
    AMGHierarchy out;
    const int L = gs_hierarchy_num_levels(h);
    for (int k = 0; k < L; ++k) {
      out.A.push_back(fetch(h, k, 0));
      if (k + 1 < L) {
        out.P.push_back(fetch(h, k, 1));
        out.R.push_back(fetch(h, k, 2));
      }
    }
    gs_hierarchy_destroy(h);
    return out;
  }

  static CsrMatrix fetch(gs_hierarchy *h, int level, int which) {
    int r = 0, c = 0, nz = 0;
    detail::check(gs_hierarchy_matrix_info(h, level, which, &r, &c, &nz));
    CsrMatrix m;
    m.nRows = r;
    m.nCols = c;
    m.rowPtr.resize(r + 1);
    m.colIdx.resize(nz);
    m.values.resize(nz);
    detail::check(gs_hierarchy_matrix(h, level, which, m.rowPtr.data(), m.colIdx.data(), m.values.data()));
    return m;
  }
  SmoothedAggregationCoarsener coarsener_;
  int maxLevels_, minDofs_;
};

}  // namespace gpuSolver
