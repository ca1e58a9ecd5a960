// gpuSolver::HostCSRMatrix (include/GPUSolver/HostSparseMatrix.h,
// src/HostSparseMatrix.cc:9-249 of the reference): a host copy of a CSR
// matrix with FP32 values and an optional symmetric permutation
// A' = P A P^T. The permuted rows come in newToOld order, every column is
// mapped by oldToNew and entries keep their order within a row (the
// reference does not re-sort them). The active arrays are the permuted ones
// once a permutation is applied, else the originals.
//
// Differences kept on purpose: the constructor from a row-major Eigen
// matrix (here: from gpuSolver::CsrMatrix, which converts from Eigen when
// it is available) copies the matrix; the reference's version builds a
// temporary and leaves the object uninitialised
// (src/HostSparseMatrix.cc:65-73). A row pointer whose last entry differs
// from nnz is refused.
#pragma once
#include <memory>

#include "Permutation.h"
#include "detail/b200.h"

namespace gpuSolver {

class HostCSRMatrix {
 public:
  HostCSRMatrix(std::size_t nRows, std::size_t nCols, std::size_t nnz, const int *rowPtr,
                const int *colIdxPtr, const float *valPtr) {
    if (nRows == 0 || nCols == 0) throw std::runtime_error("HostCSRMatrix: matrix dimensions must be nonzero.");
    if (rowPtr == nullptr || colIdxPtr == nullptr || valPtr == nullptr)
      throw std::runtime_error("HostCSRMatrix: input pointers must not be null.");
    if (rowPtr[nRows] != static_cast<int>(nnz))
      throw std::runtime_error("HostCSRMatrix: rowPtr[nRows] must equal nnz.");
    nRows_ = nRows;
    nCols_ = nCols;
    rp_.assign(rowPtr, rowPtr + nRows + 1);
    ci_.assign(colIdxPtr, colIdxPtr + nnz);
    v_.assign(valPtr, valPtr + nnz);
  }
  HostCSRMatrix(std::size_t nRows, std::size_t nCols, std::size_t nnz, const int *rowPtr,
                const int *colIdxPtr, const float *valPtr, const Permutation &permutation)
      : HostCSRMatrix(nRows, nCols, nnz, rowPtr, colIdxPtr, valPtr) {
    applyPermutation(permutation);
  }
  explicit HostCSRMatrix(const CsrMatrix &a) {
    if (a.rows() == 0 || a.cols() == 0) throw std::runtime_error("HostCSRMatrix: matrix dimensions must be nonzero.");
    nRows_ = static_cast<std::size_t>(a.rows());
    nCols_ = static_cast<std::size_t>(a.cols());
    rp_ = a.rowPtr;
    ci_ = a.colIdx;
    v_.assign(a.values.begin(), a.values.end());
  }
  HostCSRMatrix(const CsrMatrix &a, const Permutation &permutation) : HostCSRMatrix(a) {
    applyPermutation(permutation);
  }
  HostCSRMatrix(const HostCSRMatrix &) = delete;
  HostCSRMatrix &operator=(const HostCSRMatrix &) = delete;

  std::size_t rows() const { return nRows_; }
  std::size_t cols() const { return nCols_; }
  std::size_t nnz() const { return ci_.size(); }
  const int *rowPtr() const { return rp_.data(); }
  const int *colIdx() const { return ci_.data(); }
  const float *values() const { return v_.data(); }

  // A' = P A P^T (src/HostSparseMatrix.cc:118-249); replaces an earlier one.
  void applyPermutation(const Permutation &permutation) {
    if (nRows_ != nCols_) throw std::runtime_error("HostCSRMatrix::applyPermutation: matrix must be square.");
    if (permutation.size() != nRows_)
      throw std::runtime_error(
          "HostCSRMatrix::applyPermutation: permutation size does not match matrix dimensions.");
    const std::vector<double> v(v_.begin(), v_.end());
    std::vector<int> prp(nRows_ + 1), pci(ci_.size());
    std::vector<double> pv(v_.size());
    detail::check(gs_apply_permutation(static_cast<int>(nRows_), rp_.data(), ci_.data(), v.data(),
                                       permutation.oldToNew(), permutation.newToOld(), prp.data(), pci.data(),
                                       pv.data()));
    perm_.reset(new Permutation(permutation.size(), permutation.oldToNew(), permutation.newToOld()));
    prp_ = std::move(prp);
    pci_ = std::move(pci);
    pv_.assign(pv.begin(), pv.end());  // FP32 values moved, not rounded
  }
  bool isPermuted() const { return perm_ != nullptr; }
  const int *activeRowPtr() const { return perm_ ? prp_.data() : rp_.data(); }
  const int *activeColPtr() const { return perm_ ? pci_.data() : ci_.data(); }
  const float *activeValPtr() const { return perm_ ? pv_.data() : v_.data(); }
  const Permutation *permutation() const { return perm_.get(); }

 private:
  std::size_t nRows_ = 0, nCols_ = 0;
  std::vector<int> rp_, ci_, prp_, pci_;
  std::vector<float> v_, pv_;
  std::unique_ptr<Permutation> perm_;
};

namespace detail {
// The active arrays of a HostCSRMatrix with FP64 values, as the C ABI takes them.
inline std::vector<double> active_values(const HostCSRMatrix &m) {
  return std::vector<double>(m.activeValPtr(), m.activeValPtr() + m.nnz());
}
}  // namespace detail

}  // namespace gpuSolver
