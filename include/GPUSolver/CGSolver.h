// gpuSolver::CGSolver (include/GPUSolver/CGSolver.h, src/CGSolver.cc:87-306 of
// the reference): preconditioned CG on one B200. With one of the library's
// preconditioners the whole solve runs fused on the device; the operator is
// the finest matrix of the preconditioner's hierarchy (the reference passes
// the same matrix to both) and `matrix` must have its shape and nonzero
// count. With a preconditioner the caller wrote (a subclass that implements
// initialize / apply itself) the solver runs the reference's loop on the
// Backend: FP32 device objects, one encoder per iteration, the stop test on
// the host after each, as src/CGSolver.cc does.
#pragma once
#include <cmath>
#include <memory>
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
    if (solver_) detail::check(gs_solver_set_tolerance(solver_, tolerance_, static_cast<int>(maxIterations_)));
  }
  void setTolerance(float tolerance) {
    tolerance_ = tolerance;
    if (solver_) detail::check(gs_solver_set_tolerance(solver_, tolerance_, static_cast<int>(maxIterations_)));
  }
  std::size_t maxIterations() const { return maxIterations_; }
  float tolerance() const { return tolerance_; }
  std::size_t getNbOfIterations() const { return iterations_; }

  void solve(const std::vector<float> &b, std::vector<float> &x) {
    checkSizes(b.size(), x.size());
    if (pc_ != nullptr) {
      solve_on_backend(b.data(), x.data());
      return;
    }
    gs_solve_stats st;
    detail::check(gs_solver_solve_f32(solver_, b.data(), x.data(), &st));
    iterations_ = static_cast<std::size_t>(st.iterations);
  }
  void solve(const std::vector<double> &b, std::vector<double> &x) {
    checkSizes(b.size(), x.size());
    if (pc_ != nullptr) {  // the Backend is FP32, as the reference's
      std::vector<float> bf(b.begin(), b.end()), xf(x.begin(), x.end());
      solve_on_backend(bf.data(), xf.data());
      x.assign(xf.begin(), xf.end());
      return;
    }
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
    if (pc.custom()) {
      init_on_backend(backend, pc, matrix, perm);
      return;
    }
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
  // src/CGSolver.cc:17-70: the (permuted) matrix as a HostCSRMatrix and on
  // the device, then the preconditioner's initialize
  void init_on_backend(Backend &backend, Preconditioner &pc, const Matrix &matrix, const Permutation *perm) {
    n_ = matrix.rows();
    const std::vector<float> v(matrix.values.begin(), matrix.values.end());
    const std::size_t n = static_cast<std::size_t>(n_), nnz = static_cast<std::size_t>(matrix.nonZeros());
    if (perm != nullptr) {
      host_.reset(new HostCSRMatrix(n, n, nnz, matrix.rowPtr.data(), matrix.colIdx.data(), v.data(), *perm));
      perm_.reset(new Permutation(perm->size(), perm->oldToNew(), perm->newToOld()));
    } else {
      host_.reset(new HostCSRMatrix(n, n, nnz, matrix.rowPtr.data(), matrix.colIdx.data(), v.data()));
    }
    device_.reset(backend.createCSRMatrix(*host_));
    pc.initialize(backend, *host_, *device_);
    backend_ = &backend;
    pc_ = &pc;
  }

  // src/CGSolver.cc:87-306: b and x in the permuted order, r = b - A x,
  // z = M r, p = z; per iteration alpha = rho / p.Ap, x += alpha p,
  // r' = r - alpha Ap, ||r'||^2 / ||b||^2 against tol^2 (the recurrence
  // residual), z' = M r', beta = rho' / rho, p = beta p + z'. The iteration
  // count is the 0-based index of the converging iteration, maxIterations
  // when none converges; a zero right-hand side gives x = 0.
  void solve_on_backend(const float *b, float *x) {
    const std::size_t n = static_cast<std::size_t>(n_);
    std::vector<float> bp(b, b + n), xp(x, x + n);
    if (perm_) {
      const int *n2o = perm_->newToOld();
      for (std::size_t i = 0; i < n; ++i) bp[i] = b[n2o[i]], xp[i] = x[n2o[i]];
    }
    double bb = 0.0;
    for (std::size_t i = 0; i < n; ++i) bb += static_cast<double>(b[i]) * b[i];
    if (std::sqrt(bb) < 1e-12) {
      for (std::size_t i = 0; i < n; ++i) x[i] = 0.0f;
      return;
    }
    Backend &be = *backend_;
    using V = std::unique_ptr<DeviceVector>;
    using S = std::unique_ptr<DeviceScalar>;
    V xd(be.createVector(n, xp.data())), bd(be.createVector(n, bp.data())), r(be.createVector(n)),
        Ax(be.createVector(n)), z(be.createVector(n)), z1(be.createVector(n)), p(be.createVector(n)),
        Ap(be.createVector(n)), r1(be.createVector(n));
    S pAp(be.createScalar()), alpha(be.createScalar()), nalpha(be.createScalar()), beta(be.createScalar()),
        rr(be.createScalar()), bb2(be.createScalar()), rel(be.createScalar()), rho(be.createScalar()),
        rho1(be.createScalar());
    {
      std::unique_ptr<BackendEncoder> e(be.createEncoder());
      be.encodeSpmv(*e, *device_, *xd, *Ax);
      be.encodeCopy(*e, *bd, *r);
      be.encodeAxpy(*e, -1.0f, *Ax, *r);
      pc_->apply(be, *e, *r, *z);
      be.encodeCopy(*e, *z, *p);
      be.encodeDot(*e, *bd, *bd, *bb2);
      be.encodeDot(*e, *r, *z, *rho);
      be.encodeDot(*e, *r, *r, *rr);
      be.encodeScalarDivide(*e, *rr, *bb2, *rel);
      be.submitAndWait(*e);
    }
    const float tol2 = tolerance_ * tolerance_;
    const float first = rel->download();
    if (!std::isfinite(first)) throw std::runtime_error("CGSolver: initial residual is NaN/Inf — check matrix and RHS.");
    if (first < tol2) {
      iterations_ = 0;
      return;
    }
    for (std::size_t it = 0; it < maxIterations_; ++it) {
      std::unique_ptr<BackendEncoder> e(be.createEncoder());
      be.encodeSpmv(*e, *device_, *p, *Ap);
      be.encodeDot(*e, *p, *Ap, *pAp);
      be.encodeScalarDivide(*e, *rho, *pAp, *alpha);
      be.encodeAxpy(*e, *alpha, *p, *xd);
      be.encodeScalarNegate(*e, *alpha, *nalpha);
      be.encodeCopy(*e, *r, *r1);
      be.encodeAxpy(*e, *nalpha, *Ap, *r1);
      be.encodeDot(*e, *r1, *r1, *rr);
      be.encodeScalarDivide(*e, *rr, *bb2, *rel);
      pc_->apply(be, *e, *r1, *z1);
      be.encodeDot(*e, *r1, *z1, *rho1);
      be.encodeScalarDivide(*e, *rho1, *rho, *beta);
      be.encodeScale(*e, *p, *beta);
      be.encodeAxpy(*e, 1.0f, *z1, *p);
      be.submitAndWait(*e);
      const float res = rel->download();
      if (!std::isfinite(res)) throw std::runtime_error("CGSolver: solver diverged (NaN/Inf residual).");
      if (res < tol2) {
        iterations_ = it;
        break;
      }
      std::swap(rho, rho1);
      std::swap(r, r1);
      std::swap(z, z1);
      if (it + 1 == maxIterations_) iterations_ = maxIterations_;
    }
    const float *xr = xd->download();
    if (perm_) {
      const int *n2o = perm_->newToOld();
      for (std::size_t i = 0; i < n; ++i) x[n2o[i]] = xr[i];
    } else {
      for (std::size_t i = 0; i < n; ++i) x[i] = xr[i];
    }
  }

  void checkSizes(std::size_t nb, std::size_t nx) const {
    if (static_cast<int>(nb) != n_) throw std::runtime_error("CGSolver::solve: RHS size does not match matrix.");
    if (static_cast<int>(nx) != n_) throw std::runtime_error("CGSolver::solve: initial guess size does not match matrix.");
  }
  int n_ = 0;
  gs_hierarchy *h_ = nullptr;
  gs_solver *solver_ = nullptr;
  // the Backend path (a caller-written preconditioner)
  Backend *backend_ = nullptr;
  Preconditioner *pc_ = nullptr;
  std::unique_ptr<HostCSRMatrix> host_;
  std::unique_ptr<DeviceCSRMatrix> device_;
  std::unique_ptr<Permutation> perm_;
  std::size_t maxIterations_ = 1000;
  float tolerance_ = 1e-6f;
  std::size_t iterations_ = 0;
};

}  // namespace gpuSolver
