// gpuSolver block helpers (include/GPUSolver/BlockUtils.h,
// src/BlockUtils.cc:7-277 of the reference): the node permutation expanded to
// degrees of freedom, the node graph of a matrix with square blocks, and
// the inverses of the 3x3 diagonal blocks.
#pragma once
#include "HostSparseMatrix.h"
#include "Permutation.h"

namespace gpuSolver {

struct BlockGraph {
  std::vector<int> rowPtr;
  std::vector<int> colPtr;
};

// src/BlockUtils.cc:7-55: node v's component c is dof blockSize * v + c.
inline Permutation expandBlockPermutation(const Permutation &nodePermutation, std::size_t numberOfNodes,
                                          std::size_t blockSize) {
  if (nodePermutation.size() != numberOfNodes)
    throw std::runtime_error("expandBlockPermutation: permutation size does not match the number of nodes.");
  const std::size_t dofs = numberOfNodes * blockSize;
  std::vector<int> o2n(dofs), n2o(dofs);
  detail::check(gs_expand_block_permutation(static_cast<int>(numberOfNodes), static_cast<int>(blockSize),
                                            nodePermutation.oldToNew(), nodePermutation.newToOld(), o2n.data(),
                                            n2o.data()));
  return Permutation(dofs, o2n.data(), n2o.data());
}

namespace detail {
inline BlockGraph block_graph(int n, const int *rp, const int *ci, std::size_t blockSize) {
  if (blockSize == 0) throw std::runtime_error("buildBlockGraph: block size must be positive.");
  BlockGraph g;
  g.rowPtr.resize(static_cast<std::size_t>(n) / blockSize + 1);
  g.colPtr.resize(rp[n] > 0 ? static_cast<std::size_t>(rp[n]) : 1);
  int gnnz = 0;
  check(gs_block_graph(n, rp, ci, static_cast<int>(blockSize), g.rowPtr.data(), g.colPtr.data(), &gnnz));
  g.colPtr.resize(static_cast<std::size_t>(gnnz));
  return g;
}
}  // namespace detail

// src/BlockUtils.cc:58-216: node i is linked to node j != i when an entry of
// block row i lies in block column j or the reverse (sorted, no duplicates).
inline BlockGraph buildBlockGraph(const CsrMatrix &matrix, std::size_t blockSize) {
  if (matrix.rows() != matrix.cols()) throw std::runtime_error("buildBlockGraph: matrix must be square.");
  return detail::block_graph(matrix.rows(), matrix.rowPtr.data(), matrix.colIdx.data(), blockSize);
}
inline BlockGraph buildBlockGraph(const HostCSRMatrix &matrix, std::size_t blockSize) {
  if (matrix.rows() != matrix.cols()) throw std::runtime_error("buildBlockGraph: matrix must be square.");
  return detail::block_graph(static_cast<int>(matrix.rows()), matrix.activeRowPtr(), matrix.activeColPtr(),
                             blockSize);
}

// src/BlockUtils.cc:218-277: 9 values per node, row-major; throws "Block
// diagonal is not SPD." when a block has no Cholesky factor. The inverses are
// computed in FP64 and rounded to FP32 once (the reference factors in FP32).
inline std::vector<float> extractInverseDiagonalBlocks3x3(const HostCSRMatrix &matrix) {
  if (matrix.rows() % 3 != 0)
    throw std::runtime_error("3x3 block smoother requires number of DOFs divisible by 3.");
  const std::vector<double> v = detail::active_values(matrix);
  std::vector<double> d(3 * matrix.rows());
  detail::check(gs_block_inverses3x3(static_cast<int>(matrix.rows()), matrix.activeRowPtr(), matrix.activeColPtr(),
                                     v.data(), d.data()));
  return std::vector<float>(d.begin(), d.end());
}

}  // namespace gpuSolver
