// gpuSolver C++ API mirror over the gpusolver_b200 C ABI (header-only).
//
// Class names, constructor and method signatures and error behaviour follow
// the reference library (theofbraune/GPU-Conjugate-Gradient-Solver,
// include/GPUSolver/*.h) so that code written against it compiles against
// these headers and links libgpusolver_b200.so instead. Failures throw
// std::runtime_error with the library's message, as the reference does.
//
// Matrices: the reference takes Eigen::SparseMatrix<float, RowMajor>; Eigen
// is optional here. gpuSolver::CsrMatrix is the native container, and when
// <Eigen/Sparse> is available it converts from a row-major Eigen matrix.
#pragma once

#include <gpusolver_b200.h>

#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#if __has_include(<Eigen/Sparse>)
#include <Eigen/Sparse>
#define GPUSOLVER_B200_HAVE_EIGEN 1
#endif

namespace gpuSolver {
namespace detail {
inline void check(int rc) {
  if (rc != GS_OK) throw std::runtime_error(gs_last_error());
}
}  // namespace detail

// Compressed sparse row matrix (int32 indices, FP64 values).
struct CsrMatrix {
  int nRows = 0, nCols = 0;
  std::vector<int> rowPtr{0};
  std::vector<int> colIdx;
  std::vector<double> values;

  CsrMatrix() = default;
  CsrMatrix(int rows, int cols, std::vector<int> rp, std::vector<int> ci, std::vector<double> v)
      : nRows(rows), nCols(cols), rowPtr(std::move(rp)), colIdx(std::move(ci)), values(std::move(v)) {}
  template <typename S>
  CsrMatrix(int rows, int cols, const int *rp, const int *ci, const S *v)
      : nRows(rows), nCols(cols), rowPtr(rp, rp + rows + 1), colIdx(ci, ci + rp[rows]),
        values(v, v + rp[rows]) {}
#ifdef GPUSOLVER_B200_HAVE_EIGEN
  template <typename S>
  CsrMatrix(const Eigen::SparseMatrix<S, Eigen::RowMajor> &m) {  // NOLINT: implicit on purpose
    Eigen::SparseMatrix<S, Eigen::RowMajor> c = m;
    c.makeCompressed();
    *this = CsrMatrix(static_cast<int>(c.rows()), static_cast<int>(c.cols()), c.outerIndexPtr(),
                      c.innerIndexPtr(), c.valuePtr());
  }
#endif
  int rows() const { return nRows; }
  int cols() const { return nCols; }
  int nonZeros() const { return rowPtr.empty() ? 0 : rowPtr.back(); }
  gs_csr view() const { return gs_csr{nRows, nCols, rowPtr.data(), colIdx.data(), values.data()}; }
};

// include/GPUSolver/Permutation.h:10-33: (oldToNew, newToOld), validated.
class Permutation {
 public:
  Permutation(std::size_t size, const int *oldToNew, const int *newToOld) {
    if (size == 0) throw std::runtime_error("Permutation: size must be nonzero.");
    if (oldToNew == nullptr || newToOld == nullptr)
      throw std::runtime_error("Permutation: input pointers must not be null.");
    o2n_.assign(oldToNew, oldToNew + size);
    n2o_.assign(newToOld, newToOld + size);
    for (std::size_t i = 0; i < size; ++i) {
      const int j = o2n_[i];
      if (j < 0 || j >= static_cast<int>(size)) throw std::runtime_error("Permutation: oldToNew contains invalid index.");
      if (n2o_[j] != static_cast<int>(i)) throw std::runtime_error("Permutation: mappings are not inverses.");
    }
  }
  Permutation(const Permutation &) = delete;
  Permutation &operator=(const Permutation &) = delete;
  Permutation(Permutation &&) noexcept = default;
  Permutation &operator=(Permutation &&) noexcept = default;
  std::size_t size() const { return o2n_.size(); }
  const int *oldToNew() const { return o2n_.data(); }
  const int *newToOld() const { return n2o_.data(); }

 private:
  std::vector<int> o2n_, n2o_;
};

// include/GPUSolver/AMGHierarchy.h:13-21
struct AMGHierarchy {
  using Matrix = CsrMatrix;
  std::vector<Matrix> A;
  std::vector<Matrix> M;  // unused by the solvers, as in the reference
  std::vector<Matrix> P;  // P[k]: level k+1 -> level k
  std::vector<Matrix> R;  // R[k]: level k -> level k+1
  // near-nullspace modes per level; always empty here (the builder refuses modes)
#ifdef GPUSOLVER_B200_HAVE_EIGEN
  std::vector<Eigen::MatrixXf> nullspaces;
#else
  std::vector<std::vector<float>> nullspaces;
#endif
  std::size_t levels() const { return A.size(); }
};

// Optional knobs of this implementation (no reference counterpart). The
// defaults reproduce the reference: smoother steps on the coarsest level and
// its V-cycle bit for bit; fast() selects the FP32 V-cycle, flexible CG,
// CUDA-graph replay, the textbook V-cycle, a dense Cholesky coarse solve (its
// packed inverse in FP16 tiles applied on the tensor cores), the smallest-last
// colouring (strong couplings only on the coarse scalar levels) and half
// sweeps.
struct B200Options {
  int precision = 0;        // 0 FP64 V-cycle, 1 FP32 V-cycle
  int flexible = 0;         // 1 Polak-Ribiere outer CG
  int useGraph = 0;         // 1 CUDA-graph replay with a device-side stop flag
  int coarseSolver = 0;     // 0 smoother steps (the reference), 1 dense Cholesky
  int referenceVCycle = 1;  // 1 the reference's V-cycle including its buffer aliasing
  int coarseRows = 0;       // > 0: dense coarsest solve on the first level with at most this many rows
  int coloring = 0;         // 0 the reference's greedy colouring, 1 smallest-last where it uses fewer colours,
                            // 2 and strong-coupling colourings of the coarse scalar levels
  int overlapLaunch = 2;    // 2 programmatic dependent launch of V-cycle kernels, graphs too; 1 eager only
  int packedRows = 8192;    // dense coarsest levels above this keep a tiled lower triangle of the inverse
  int sweepLaunch = 1;      // 0 one launch per colour pass, 1 cooperative sweeps where faster, 2 always
  int halfSweeps = 0;       // 1 forward sweeps before and backward sweeps after the coarse correction
  int coarseHalf = 0;       // 1 packed dense coarsest inverse in FP16 tiles (tensor-core apply)
  static B200Options fast() {
    B200Options o;
    o.precision = 1;
    o.flexible = 1;
    o.useGraph = 1;
    o.coarseSolver = 1;
    o.referenceVCycle = 0;
    o.coarseRows = 24576;
    o.coloring = 2;
    o.halfSweeps = 1;
    o.coarseHalf = 1;
    return o;
  }
};

}  // namespace gpuSolver
