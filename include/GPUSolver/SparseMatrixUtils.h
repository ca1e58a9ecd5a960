// gpuSolver::permuteMatrix (include/GPUSolver/SparseMatrixUtils.h,
// src/SparseMatrixUtils.cc:8-31 of the reference): entry (i, j) moves to
// (rowOldToNew[i], colOldToNew[j]); the result has its columns sorted within
// each row, as Eigen's setFromTriplets leaves them. Both maps must be
// permutations of their index range. The reference takes and returns a
// row-major Eigen matrix; here the container is gpuSolver::CsrMatrix (built
// from Eigen implicitly when Eigen is available).
#pragma once
#include "detail/b200.h"

namespace gpuSolver {

inline CsrMatrix permuteMatrix(const CsrMatrix &M, const int *rowOldToNew, const int *colOldToNew) {
  CsrMatrix out;
  out.nRows = M.rows();
  out.nCols = M.cols();
  out.rowPtr.assign(static_cast<std::size_t>(M.rows()) + 1, 0);
  out.colIdx.resize(static_cast<std::size_t>(M.nonZeros()));
  out.values.resize(static_cast<std::size_t>(M.nonZeros()));
  detail::check(gs_permute_matrix(M.rows(), M.cols(), M.rowPtr.data(), M.colIdx.data(), M.values.data(),
                                  rowOldToNew, colOldToNew, out.rowPtr.data(), out.colIdx.data(),
                                  out.values.data()));
  return out;
}

}  // namespace gpuSolver
