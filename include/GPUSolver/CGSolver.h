// gpuSolver::CGSolver (include/GPUSolver/CGSolver.h, src/CGSolver.cc:87-306 of
// the reference): preconditioned CG on one B200. The operator is the finest
// matrix of the preconditioner's hierarchy (the reference passes the same
// matrix to both); `matrix` must have its shape and nonzero count.
#pragma once
#include <vector>

#include "Preconditioner.h"

namespace gpuSolver {

class CGSolver {
 public:
  using Matrix = CsrMatrix;

  CGSolver(Backend &backend, Preconditioner &preconditioner, const Matrix &matrix)
      : CGSolver(backend, preconditioner, matrix, nullptr) {}
  CGSolver(Backend &backend, Preconditioner &preconditioner, const Matrix &matrix,
           const Permutation &permutationForMatrix)
      : CGSolver(backend, preconditioner, matrix, &permutationForMatrix) {}
  ~CGSolver() {
    if (solver_) gs_solver_destroy(solver_);
    if (h_) gs_hierarchy_destroy(h_);
  }
  CGSolver(const CGSolver &) = delete;
  CGSolver &operator=(const CGSolver &) = delete;

  void setMaxIterations(std::size_t maxIterations) {
    maxIterations_ = maxIterations;
    detail::check(gs_solver_set_tolerance(solver_, tolerance_, static_cast<int>(maxIterations_)));
  }
  void setTolerance(float tolerance) {
    tolerance_ = tolerance;
    detail::check(gs_solver_set_tolerance(solver_, tolerance_, static_cast<int>(maxIterations_)));
  }
  std::size_t maxIterations() const { return maxIterations_; }
  float tolerance() const { return tolerance_; }
  std::size_t getNbOfIterations() const { return iterations_; }

  void solve(const std::vector<float> &b, std::vector<float> &x) {
    checkSizes(b.size(), x.size());
    gs_solve_stats st;
    detail::check(gs_solver_solve_f32(solver_, b.data(), x.data(), &st));
    iterations_ = static_cast<std::size_t>(st.iterations);
  }
  void solve(const std::vector<double> &b, std::vector<double> &x) {
    checkSizes(b.size(), x.size());
    gs_solve_stats st;
    detail::check(gs_solver_solve(solver_, b.data(), x.data(), &st));
    iterations_ = static_cast<std::size_t>(st.iterations);
  }
#ifdef GPUSOLVER_B200_HAVE_EIGEN
  void solve(const Eigen::VectorXf &b, Eigen::VectorXf &x) {
    std::vector<float> bv(b.data(), b.data() + b.size()), xv(x.data(), x.data() + x.size());
    solve(bv, xv);
    for (Eigen::Index i = 0; i < x.size(); ++i) x[i] = xv[static_cast<std::size_t>(i)];
  }
#endif

 private:
  CGSolver(Backend &backend, Preconditioner &pc, const Matrix &matrix, const Permutation *perm) {
    if (matrix.rows() == 0 || matrix.cols() == 0) throw std::runtime_error("CGSolver: matrix must be non-empty.");
    if (matrix.rows() != matrix.cols()) throw std::runtime_error("CGSolver: matrix must be square.");
    if (pc.singleLevel()) {
      init_single_level(backend, pc, matrix, perm);
      return;
    }
    const AMGHierarchy &H = pc.hierarchy();
    if (H.A[0].rows() != matrix.rows() || H.A[0].nonZeros() != matrix.nonZeros())
      throw std::runtime_error("CGSolver: matrix does not match the preconditioner's finest level.");
    if (perm != nullptr && perm->size() != static_cast<std::size_t>(matrix.rows()))
      throw std::runtime_error(" the permutation is incompatible with the passed vectors");
    n_ = matrix.rows();
    std::vector<gs_csr> A, P, R;
    for (const auto &m : H.A) A.push_back(m.view());
    for (const auto &m : H.P) P.push_back(m.view());
    for (const auto &m : H.R) R.push_back(m.view());
    detail::check(gs_hierarchy_from_levels(static_cast<int>(A.size()), A.data(), P.data(), R.data(),
                                           pc.blockSize(), &h_));
    std::vector<const int *> o2n, n2o;
    for (const Permutation &p : pc.permutations()) o2n.push_back(p.oldToNew()), n2o.push_back(p.newToOld());
    if (perm != nullptr) o2n[0] = perm->oldToNew(), n2o[0] = perm->newToOld();
    gs_solver_options opt = pc.options();
    opt.tol = tolerance_;
    opt.max_iter = static_cast<int>(maxIterations_);
    detail::check(gs_solver_create(h_, o2n.data(), n2o.data(), &opt, backend.device(), &solver_));
  }
  // a one-level hierarchy of the CG's matrix, smoothed from zero
  void init_single_level(Backend &backend, Preconditioner &pc, const Matrix &matrix, const Permutation *perm) {
    n_ = matrix.rows();
    if (perm != nullptr && perm->size() != static_cast<std::size_t>(n_))
      throw std::runtime_error(" the permutation is incompatible with the passed vectors");
    const gs_csr a = matrix.view();
    detail::check(gs_hierarchy_from_levels(1, &a, nullptr, nullptr, pc.blockSize(), &h_));
    const int *o2n = perm ? perm->oldToNew() : nullptr;
    const int *n2o = perm ? perm->newToOld() : nullptr;
    gs_solver_options opt = pc.options();
    opt.tol = tolerance_;
    opt.max_iter = static_cast<int>(maxIterations_);
    detail::check(gs_solver_create(h_, perm ? &o2n : nullptr, perm ? &n2o : nullptr, &opt, backend.device(), &solver_));
  }
  void checkSizes(std::size_t nb, std::size_t nx) const {
    if (static_cast<int>(nb) != n_) throw std::runtime_error("CGSolver::solve: RHS size does not match matrix.");
    if (static_cast<int>(nx) != n_) throw std::runtime_error("CGSolver::solve: initial guess size does not match matrix.");
  }
  int n_ = 0;
  gs_hierarchy *h_ = nullptr;
  gs_solver *solver_ = nullptr;
  std::size_t maxIterations_ = 1000;
  float tolerance_ = 1e-6f;
  std::size_t iterations_ = 0;
};

}  // namespace gpuSolver
