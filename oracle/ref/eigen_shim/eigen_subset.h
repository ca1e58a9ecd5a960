// Test infrastructure only (oracle). Not part of the shipped library.
//
// A minimal, project-written stand-in for the small subset of the Eigen API
// that the reference's solver layer uses, so that the reference's own
// sources (CGSolver.cc, MultigridSmoother.cc, SparseMatrixUtils.cc,
// BlockUtils.cc, HostSparseMatrix.cc, the smoothers and preconditioners)
// compile unmodified, in place, into the reference oracle `oracle/_ref/`.
//
// Eigen itself is not installed in this image. The reference pins Eigen at
// 6aebfa9acc529f8622fb6eb063ebee8db59be0c5 (cmake/recipes/eigen.cmake:29).
// Only the following are provided, with the semantics the reference relies on:
//   * SparseMatrix<float, RowMajor>: compressed CSR; setFromTriplets sorts
//     columns within each row and sums duplicates in input order
//     (used by permuteMatrix, src/SparseMatrixUtils.cc:8-31);
//     InnerIterator; outer/inner/value pointers.
//   * Matrix<S, R, C>: dense column-major storage with VectorXf, MatrixXf,
//     Matrix3f typedefs; norm(), setZero(), Zero(), Identity().
//   * LLT<Matrix3f>: textbook Cholesky (lower), used only by
//     extractInverseDiagonalBlocks3x3 (src/BlockUtils.cc:218-277). Its
//     rounding is not Eigen's, so the 3x3 inverse blocks agree with real
//     Eigen only to FP32 rounding, not bit for bit.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace Eigen {

using Index = std::ptrdiff_t;
enum StorageOptions { ColMajor = 0, RowMajor = 1 };
enum ComputationInfo { Success = 0, NumericalIssue = 1 };
constexpr int Dynamic = -1;

template <typename S, int R, int C>
class Matrix {
 public:
  using Scalar = S;
  Matrix() : rows_(R > 0 ? R : 0), cols_(C > 0 ? C : 0), data_(rows_ * cols_, S(0)) {}
  explicit Matrix(Index n) : rows_(R == 1 ? 1 : n), cols_(R == 1 ? n : (C > 0 ? C : 1)) {
    data_.assign(rows_ * cols_, S(0));
  }
  Matrix(Index r, Index c) : rows_(r), cols_(c), data_(r * c, S(0)) {}

  Index rows() const { return rows_; }
  Index cols() const { return cols_; }
  Index size() const { return rows_ * cols_; }
  S *data() { return data_.data(); }
  const S *data() const { return data_.data(); }

  S &operator()(Index i) { return data_[i]; }
  const S &operator()(Index i) const { return data_[i]; }
  S &operator[](Index i) { return data_[i]; }
  const S &operator[](Index i) const { return data_[i]; }
  S &operator()(Index r, Index c) { return data_[c * rows_ + r]; }
  const S &operator()(Index r, Index c) const { return data_[c * rows_ + r]; }

  void setZero() { std::fill(data_.begin(), data_.end(), S(0)); }
  void resize(Index n) { rows_ = (C == 1 ? n : 1); cols_ = (C == 1 ? 1 : n); data_.assign(n, S(0)); }

  S squaredNorm() const {
    double acc = 0.0;
    for (const S &v : data_) acc += double(v) * double(v);
    return S(acc);
  }
  S norm() const { return S(std::sqrt(double(squaredNorm()))); }

  static Matrix Zero() { return Matrix(); }
  static Matrix Zero(Index n) { return Matrix(n); }
  static Matrix Zero(Index r, Index c) { return Matrix(r, c); }
  static Matrix Identity() {
    Matrix m;
    for (Index i = 0; i < std::min(m.rows_, m.cols_); ++i) m(i, i) = S(1);
    return m;
  }
  static Matrix Identity(Index r, Index c) {
    Matrix m(r, c);
    for (Index i = 0; i < std::min(r, c); ++i) m(i, i) = S(1);
    return m;
  }

 private:
  Index rows_, cols_;
  std::vector<S> data_;
};

using VectorXf = Matrix<float, Dynamic, 1>;
using VectorXd = Matrix<double, Dynamic, 1>;
using MatrixXf = Matrix<float, Dynamic, Dynamic>;
using Matrix3f = Matrix<float, 3, 3>;

template <typename MatrixType>
class LLT {
 public:
  using S = typename MatrixType::Scalar;
  explicit LLT(const MatrixType &a) : l_(a.rows(), a.cols()), info_(Success) {
    const Index n = a.rows();
    for (Index j = 0; j < n; ++j) {
      S d = a(j, j);
      for (Index k = 0; k < j; ++k) d -= l_(j, k) * l_(j, k);
      if (!(d > S(0))) { info_ = NumericalIssue; return; }
      const S ljj = std::sqrt(d);
      l_(j, j) = ljj;
      for (Index i = j + 1; i < n; ++i) {
        S s = a(i, j);
        for (Index k = 0; k < j; ++k) s -= l_(i, k) * l_(j, k);
        l_(i, j) = s / ljj;
      }
    }
  }
  ComputationInfo info() const { return info_; }
  MatrixType solve(const MatrixType &b) const {
    const Index n = l_.rows();
    MatrixType x = b;
    for (Index c = 0; c < b.cols(); ++c) {
      for (Index i = 0; i < n; ++i) {  // L y = b
        S s = x(i, c);
        for (Index k = 0; k < i; ++k) s -= l_(i, k) * x(k, c);
        x(i, c) = s / l_(i, i);
      }
      for (Index i = n - 1; i >= 0; --i) {  // L^T x = y
        S s = x(i, c);
        for (Index k = i + 1; k < n; ++k) s -= l_(k, i) * x(k, c);
        x(i, c) = s / l_(i, i);
      }
    }
    return x;
  }

 private:
  MatrixType l_;
  ComputationInfo info_;
};

template <typename S>
class Triplet {
 public:
  Triplet(Index r, Index c, S v) : r_(r), c_(c), v_(v) {}
  Index row() const { return r_; }
  Index col() const { return c_; }
  const S &value() const { return v_; }

 private:
  Index r_, c_;
  S v_;
};

template <typename S, int Options = ColMajor>
class SparseMatrix {
  static_assert(Options == RowMajor, "the shim provides row-major storage only");

 public:
  using Scalar = S;
  SparseMatrix() : rows_(0), cols_(0), outer_(1, 0) {}
  SparseMatrix(Index r, Index c) : rows_(r), cols_(c), outer_(r + 1, 0) {}

  Index rows() const { return rows_; }
  Index cols() const { return cols_; }
  Index outerSize() const { return rows_; }
  Index nonZeros() const { return static_cast<Index>(inner_.size()); }
  void makeCompressed() {}

  int *outerIndexPtr() { return outer_.data(); }
  const int *outerIndexPtr() const { return outer_.data(); }
  int *innerIndexPtr() { return inner_.data(); }
  const int *innerIndexPtr() const { return inner_.data(); }
  S *valuePtr() { return values_.data(); }
  const S *valuePtr() const { return values_.data(); }

  // Builds the matrix from raw CSR arrays (a shim-only helper used by the
  // oracle's C entry points to hand data to the reference code).
  void assignCsr(Index r, Index c, const int *rowPtr, const int *col, const S *val) {
    rows_ = r;
    cols_ = c;
    outer_.assign(rowPtr, rowPtr + r + 1);
    inner_.assign(col, col + rowPtr[r]);
    values_.assign(val, val + rowPtr[r]);
  }

  template <typename It>
  void setFromTriplets(It begin, It end) {
    std::vector<std::size_t> order;
    std::vector<Index> rr, cc;
    std::vector<S> vv;
    for (It it = begin; it != end; ++it) {
      rr.push_back(it->row());
      cc.push_back(it->col());
      vv.push_back(it->value());
    }
    order.resize(rr.size());
    std::iota(order.begin(), order.end(), std::size_t(0));
    std::stable_sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) {
      return rr[a] != rr[b] ? rr[a] < rr[b] : cc[a] < cc[b];
    });
    outer_.assign(rows_ + 1, 0);
    inner_.clear();
    values_.clear();
    for (std::size_t k = 0; k < order.size(); ++k) {
      const std::size_t t = order[k];
      if (k > 0) {
        const std::size_t p = order[k - 1];
        if (rr[p] == rr[t] && cc[p] == cc[t]) {
          values_.back() += vv[t];
          continue;
        }
      }
      inner_.push_back(static_cast<int>(cc[t]));
      values_.push_back(vv[t]);
      outer_[rr[t] + 1]++;
    }
    for (Index i = 0; i < rows_; ++i) outer_[i + 1] += outer_[i];
  }

  class InnerIterator {
   public:
    InnerIterator(const SparseMatrix &m, Index outer)
        : m_(m), row_(outer), k_(m.outer_[outer]), end_(m.outer_[outer + 1]) {}
    explicit operator bool() const { return k_ < end_; }
    InnerIterator &operator++() { ++k_; return *this; }
    Index row() const { return row_; }
    Index col() const { return m_.inner_[k_]; }
    Index index() const { return m_.inner_[k_]; }
    const S &value() const { return m_.values_[k_]; }

   private:
    const SparseMatrix &m_;
    Index row_;
    int k_, end_;
  };

 private:
  Index rows_, cols_;
  std::vector<int> outer_;
  std::vector<int> inner_;
  std::vector<S> values_;
};

}  // namespace Eigen
