// gpuSolver::HostELLMatrix (include/GPUSolver/HostELLMatrix.h,
// src/HostELLMatrix.cc:10-206 of the reference): the active arrays of a
// HostCSRMatrix as an ELL part of ellWidth slots, stored slot-major
// (index = slot * rows + row; padding column 0, value 0), plus the entries
// past the width of each row as an overflow CSR.
#pragma once
#include "HostSparseMatrix.h"

namespace gpuSolver {

class HostELLMatrix {
 public:
  HostELLMatrix(const HostCSRMatrix &csr, std::size_t ellWidth)
      : nRows_(csr.rows()), nCols_(csr.cols()), nnz_(csr.nnz()), width_(ellWidth) {
    if (nRows_ == 0 || nCols_ == 0) throw std::runtime_error("HostELLMatrix: matrix dimensions must be nonzero.");
    if (ellWidth == 0) throw std::runtime_error("HostELLMatrix: ELL width must be nonzero.");
    const std::vector<double> v = detail::active_values(csr);
    const std::size_t cells = nRows_ * width_;
    std::vector<double> ev(cells), ov(nnz_ > 0 ? nnz_ : 1);
    ellCol_.resize(cells);
    ovfRowPtr_.resize(nRows_ + 1);
    ovfCol_.resize(nnz_ > 0 ? nnz_ : 1);
    int ovf = 0;
    detail::check(gs_ell_build(static_cast<int>(nRows_), static_cast<int>(nCols_), csr.activeRowPtr(),
                               csr.activeColPtr(), v.data(), static_cast<int>(width_), ellCol_.data(), ev.data(),
                               ovfRowPtr_.data(), ovfCol_.data(), ov.data(), &ovf));
    ellVal_.assign(ev.begin(), ev.end());
    ovfCol_.resize(static_cast<std::size_t>(ovf));
    ovfVal_.assign(ov.begin(), ov.begin() + ovf);
  }
  HostELLMatrix(const HostELLMatrix &) = delete;
  HostELLMatrix &operator=(const HostELLMatrix &) = delete;

  std::size_t rows() const { return nRows_; }
  std::size_t cols() const { return nCols_; }
  std::size_t nnz() const { return nnz_; }
  std::size_t ellWidth() const { return width_; }
  std::size_t overflowNnz() const { return ovfCol_.size(); }
  const int *ellColIdx() const { return ellCol_.data(); }
  const float *ellValues() const { return ellVal_.data(); }
  const int *overflowRowPtr() const { return ovfRowPtr_.data(); }
  const int *overflowColIdx() const { return ovfCol_.data(); }
  const float *overflowValues() const { return ovfVal_.data(); }

 private:
  std::size_t nRows_, nCols_, nnz_, width_;
  std::vector<int> ellCol_, ovfRowPtr_, ovfCol_;
  std::vector<float> ellVal_, ovfVal_;
};

}  // namespace gpuSolver
