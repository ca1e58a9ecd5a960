// Test infrastructure only (oracle). Not part of the shipped library.
//
// C entry points into the reference's own CPU implementation, compiled
// unmodified from the reference source tree (see oracle/ref/Makefile) against
// the project-written Eigen subset in oracle/ref/eigen_shim. Python tests load
// the resulting oracle/_ref/libgsref.so through ctypes to
//   * generate golden vectors (tests/golden/make_golden.py),
//   * pin the project's CPU restatement (oracle/oracle.cc) against the
//     reference bit for bit in FP32, and
//   * time the reference CPU path as the reported CPU baseline (bench.py).
// Every function returns 0 on success and -1 when the reference threw; the
// message is then available from gsref_last_error().

#include <GPUSolver/AMGHierarchy.h>
#include <GPUSolver/Backend.h>
#include <GPUSolver/BackendEncoder.h>
#include <GPUSolver/BlockUtils.h>
#include <GPUSolver/CGSolver.h>
#include <GPUSolver/CPU/CPUBackend.h>
#include <GPUSolver/CPU/CPUDeviceIndexVector.h>
#include <GPUSolver/DeviceScalar.h>
#include <GPUSolver/DeviceSparseMatrix.h>
#include <GPUSolver/DeviceVector.h>
#include <GPUSolver/GraphColoring.h>
#include <GPUSolver/HostELLMatrix.h>
#include <GPUSolver/HostSparseMatrix.h>
#include <GPUSolver/Permutation.h>
#include <GPUSolver/Preconditioners/IdentityPreconditioner.h>
#include <GPUSolver/Preconditioners/JacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridBlockGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/SymmetricGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/BlockGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/BlockJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/DampedJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridBlockJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridDampedJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridHybridBlockPreconditioner.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <GPUSolver/SparseMatrixUtils.h>
#include <iostream>
#include <GPUSolver/ReorderingStrategies/HierarchicalReordering.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_last_error;

using SpMat = Eigen::SparseMatrix<float, Eigen::RowMajor>;

SpMat make_matrix(int rows, int cols, const int *rowptr, const int *col, const float *val) {
  SpMat m;
  m.assignCsr(rows, cols, rowptr, col, val);
  return m;
}

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // namespace

// The reference prints diagnostics through std::cout (e.g. orphan rows in
// HierarchicalReordering); this library carries its own copy of the C++
// runtime, so its standard streams are initialised here explicitly.
static std::ios_base::Init g_streams_ready;

extern "C" {

// Plain CSR view used by the hierarchy entry points below.
struct gsref_csr {
  int rows, cols;
  const int *rowptr;
  const int *col;
  const float *val;
};

const char *gsref_last_error() { return g_last_error.c_str(); }

int gsref_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void gsref_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// GraphColoring::compute (src/GraphColoring.cc:9-72).
int gsref_coloring(int n, const int *rowptr, const int *col, int *colors, int *color_vertices,
                   int *color_offsets, int *ncolors) {
  return guarded([&] {
    gpuSolver::GraphColoring c;
    c.compute(static_cast<std::size_t>(n), rowptr, col);
    *ncolors = static_cast<int>(c.numberOfColors());
    std::memcpy(colors, c.colors().data(), sizeof(int) * n);
    std::memcpy(color_vertices, c.colorVertices().data(), sizeof(int) * n);
    std::memcpy(color_offsets, c.colorOffsets().data(), sizeof(int) * (*ncolors + 1));
  });
}

// RCMReordering::compute (src/ReorderingStrategies/RCMReordering.cc:11-110).
int gsref_rcm(int n, const int *rowptr, const int *col, int *old_to_new, int *new_to_old) {
  return guarded([&] {
    gpuSolver::RCMReordering rcm;
    rcm.compute(static_cast<std::size_t>(n), rowptr, col, old_to_new, new_to_old);
  });
}

// HostCSRMatrix::applyPermutation (src/HostSparseMatrix.cc:118-249).
int gsref_apply_permutation(int n, const int *rowptr, const int *col, const float *val,
                            const int *old_to_new, const int *new_to_old, int *out_rowptr,
                            int *out_col, float *out_val) {
  return guarded([&] {
    gpuSolver::Permutation p(n, old_to_new, new_to_old);
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val, p);
    std::memcpy(out_rowptr, m.activeRowPtr(), sizeof(int) * (n + 1));
    std::memcpy(out_col, m.activeColPtr(), sizeof(int) * rowptr[n]);
    std::memcpy(out_val, m.activeValPtr(), sizeof(float) * rowptr[n]);
  });
}

// permuteMatrix (src/SparseMatrixUtils.cc:8-31).
int gsref_permute_matrix(int rows, int cols, const int *rowptr, const int *col, const float *val,
                         const int *row_old_to_new, const int *col_old_to_new, int *out_rowptr,
                         int *out_col, float *out_val) {
  return guarded([&] {
    SpMat m = make_matrix(rows, cols, rowptr, col, val);
    SpMat r = gpuSolver::permuteMatrix(m, row_old_to_new, col_old_to_new);
    std::memcpy(out_rowptr, r.outerIndexPtr(), sizeof(int) * (rows + 1));
    std::memcpy(out_col, r.innerIndexPtr(), sizeof(int) * r.nonZeros());
    std::memcpy(out_val, r.valuePtr(), sizeof(float) * r.nonZeros());
  });
}

// HostELLMatrix constructor (src/HostELLMatrix.cc:10-206). The overflow
// arrays must hold nnz entries (an upper bound).
int gsref_ell(int n, const int *rowptr, const int *col, const float *val, int width,
              int *ell_col, float *ell_val, int *ovf_rowptr, int *ovf_col, float *ovf_val,
              int *ovf_nnz) {
  return guarded([&] {
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    gpuSolver::HostELLMatrix e(m, width);
    std::memcpy(ell_col, e.ellColIdx(), sizeof(int) * n * width);
    std::memcpy(ell_val, e.ellValues(), sizeof(float) * n * width);
    std::memcpy(ovf_rowptr, e.overflowRowPtr(), sizeof(int) * (n + 1));
    *ovf_nnz = static_cast<int>(e.overflowNnz());
    if (e.overflowNnz() > 0) {
      std::memcpy(ovf_col, e.overflowColIdx(), sizeof(int) * e.overflowNnz());
      std::memcpy(ovf_val, e.overflowValues(), sizeof(float) * e.overflowNnz());
    }
  });
}

// CPUBackend::encodeSpmv (src/CPU/CPUBackend.cc:217-236).
int gsref_spmv(int rows, int cols, const int *rowptr, const int *col, const float *val,
               const float *x, float *y) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    gpuSolver::HostCSRMatrix m(rows, cols, rowptr[rows], rowptr, col, val);
    std::unique_ptr<gpuSolver::DeviceCSRMatrix> A(be.createCSRMatrix(m));
    std::unique_ptr<gpuSolver::DeviceVector> xv(be.createVector(cols, x));
    std::unique_ptr<gpuSolver::DeviceVector> yv(be.createVector(rows));
    be.spmv(*A, *xv, *yv);
    std::memcpy(y, yv->download(), sizeof(float) * rows);
  });
}

// CPUBackend::encodeGaussSeidelColor (src/CPU/CPUBackend.cc:238-268): one
// color pass over color_vertices[start, start + count), in place on x.
int gsref_gs_color(int n, const int *rowptr, const int *col, const float *val,
                   const int *color_vertices, int nvertices, int start, int count,
                   const float *rhs, float *x, float omega) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    std::unique_ptr<gpuSolver::DeviceCSRMatrix> A(be.createCSRMatrix(m));
    gpuSolver::CPUDeviceIndexVector order(nvertices, color_vertices);
    std::unique_ptr<gpuSolver::DeviceVector> b(be.createVector(n, rhs));
    std::unique_ptr<gpuSolver::DeviceVector> xv(be.createVector(n, x));
    std::unique_ptr<gpuSolver::BackendEncoder> enc(be.createEncoder());
    be.encodeGaussSeidelColor(*enc, *A, order, start, count, *b, *xv, omega);
    be.submitAndWait(*enc);
    std::memcpy(x, xv->download(), sizeof(float) * n);
  });
}

// CPUBackend::encodeApplyBlockInverses3x3 (src/CPU/CPUBackend.cc:323-348).
int gsref_apply_block_inverses3x3(int n, const float *dinv, const float *r, float *c) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    std::unique_ptr<gpuSolver::DeviceVector> d(be.createVector(3 * n, dinv));
    std::unique_ptr<gpuSolver::DeviceVector> rv(be.createVector(n, r));
    std::unique_ptr<gpuSolver::DeviceVector> cv(be.createVector(n));
    std::unique_ptr<gpuSolver::BackendEncoder> enc(be.createEncoder());
    be.encodeApplyBlockInverses3x3(*enc, *d, *rv, *cv);
    std::memcpy(c, cv->download(), sizeof(float) * n);
  });
}

// CPUBackend::encodeBlockGaussSeidelColor3x3 (src/CPU/CPUBackend.cc:350-387).
// The reference reads its fifth argument as an END index (see
// src/CPU/CPUBackend.cc:364); this entry point passes `end` straight through.
int gsref_block_gs_color3x3(int n, const int *rowptr, const int *col, const float *val,
                            const int *color_blocks, int nblocks, int begin, int end,
                            const float *dinv, const float *rhs, float *x, float omega) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    std::unique_ptr<gpuSolver::DeviceCSRMatrix> A(be.createCSRMatrix(m));
    gpuSolver::CPUDeviceIndexVector order(nblocks, color_blocks);
    std::unique_ptr<gpuSolver::DeviceVector> d(be.createVector(3 * n, dinv));
    std::unique_ptr<gpuSolver::DeviceVector> b(be.createVector(n, rhs));
    std::unique_ptr<gpuSolver::DeviceVector> xv(be.createVector(n, x));
    std::unique_ptr<gpuSolver::BackendEncoder> enc(be.createEncoder());
    be.encodeBlockGaussSeidelColor3x3(*enc, *A, order, *d, begin, end, *b, *xv, omega);
    std::memcpy(x, xv->download(), sizeof(float) * n);
  });
}

// extractInverseDiagonalBlocks3x3 (src/BlockUtils.cc:218-277).
int gsref_block_inverses3x3(int n, const int *rowptr, const int *col, const float *val,
                            float *dinv) {
  return guarded([&] {
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    std::vector<float> inv = gpuSolver::extractInverseDiagonalBlocks3x3(m);
    std::memcpy(dinv, inv.data(), sizeof(float) * inv.size());
  });
}

// buildBlockGraph (src/BlockUtils.cc:126-216); colptr holds up to nnz entries.
int gsref_block_graph(int n, const int *rowptr, const int *col, const float *val, int *g_rowptr,
                      int *g_col) {
  return guarded([&] {
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    gpuSolver::BlockGraph g = gpuSolver::buildBlockGraph(m, 3);
    std::memcpy(g_rowptr, g.rowPtr.data(), sizeof(int) * g.rowPtr.size());
    std::memcpy(g_col, g.colPtr.data(), sizeof(int) * g.colPtr.size());
  });
}

// CPUBackend::encodeDot (src/CPU/CPUBackend.cc:269-284).
int gsref_dot(int n, const float *x, const float *y, float *out) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    std::unique_ptr<gpuSolver::DeviceVector> xv(be.createVector(n, x));
    std::unique_ptr<gpuSolver::DeviceVector> yv(be.createVector(n, y));
    std::unique_ptr<gpuSolver::DeviceScalar> s(be.createScalar());
    be.dot(*xv, *yv, *s);
    *out = s->download();
  });
}

// SymmetricGaussSeidelPreconditioner::apply (zero initial guess, `sweeps`
// symmetric steps) on one matrix in its given order.
int gsref_sgs_apply(int n, const int *rowptr, const int *col, const float *val,
                    const float *rhs, float *z, float omega, int sweeps) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    gpuSolver::HostCSRMatrix m(n, n, rowptr[n], rowptr, col, val);
    std::unique_ptr<gpuSolver::DeviceCSRMatrix> A(be.createCSRMatrix(m));
    gpuSolver::SymmetricGaussSeidelPreconditioner pc(omega, sweeps);
    pc.initialize(be, m, *A);
    std::unique_ptr<gpuSolver::DeviceVector> b(be.createVector(n, rhs));
    std::unique_ptr<gpuSolver::DeviceVector> zv(be.createVector(n));
    std::unique_ptr<gpuSolver::BackendEncoder> enc(be.createEncoder());
    pc.apply(be, *enc, *b, *zv);
    std::memcpy(z, zv->download(), sizeof(float) * n);
  });
}

// The reference's AMG-PCG path end to end: AMGHierarchy + per-level
// permutations -> Multigrid{GaussSeidel,BlockGaussSeidel}Preconditioner ->
// CGSolver(backend, preconditioner, A0, permutation[0]) -> solve(b, x).
//   smoother: 0 = MultigridGaussSeidelPreconditioner (coarse steps =
//             pre + post, src/Preconditioners/MultigridGaussSeidelPreconditioner.cc:21),
//             1 = MultigridBlockGaussSeidelPreconditioner (coarse steps given),
//             2 = MultigridDampedJacobiPreconditioner (coarse steps = pre + post),
//             3 = MultigridBlockJacobiPreconditioner, 4 = MultigridHybridBlockPreconditioner
//             (block GS on the finest level, block Jacobi below; coarse steps given).
//   perms: per level, old_to_new then new_to_old (each n_k ints); NULL means
//          identity on every level.
// `x` holds the initial guess on entry and the result on exit. `solve_ms`
// receives the wall time of CGSolver::solve alone; `setup_ms` the time of the
// preconditioner and solver construction.
int gsref_amg_pcg(int nlevels, const gsref_csr *A, const gsref_csr *P, const gsref_csr *R,
                  const int *const *perm_old_to_new, const int *const *perm_new_to_old,
                  int smoother, int pre, int post, int coarse, int vcycles, float omega,
                  float tol, int max_iter, const float *b, float *x, int *iterations,
                  double *setup_ms, double *solve_ms) {
  return guarded([&] {
    using Clock = std::chrono::steady_clock;
    gpuSolver::AMGHierarchy h;
    for (int k = 0; k < nlevels; ++k) {
      h.A.push_back(make_matrix(A[k].rows, A[k].cols, A[k].rowptr, A[k].col, A[k].val));
      if (k + 1 < nlevels) {
        h.P.push_back(make_matrix(P[k].rows, P[k].cols, P[k].rowptr, P[k].col, P[k].val));
        h.R.push_back(make_matrix(R[k].rows, R[k].cols, R[k].rowptr, R[k].col, R[k].val));
      }
    }
    std::vector<gpuSolver::Permutation> perms;
    for (int k = 0; k < nlevels; ++k) {
      const int n = A[k].rows;
      if (perm_old_to_new != nullptr) {
        perms.emplace_back(n, perm_old_to_new[k], perm_new_to_old[k]);
      } else {
        std::vector<int> id(n);
        for (int i = 0; i < n; ++i) id[i] = i;
        perms.emplace_back(n, id.data(), id.data());
      }
    }
    const int n0 = A[0].rows;
    gpuSolver::CPUBackend be;
    auto t0 = Clock::now();
    std::unique_ptr<gpuSolver::Preconditioner> pc;
    if (smoother == 0) {
      pc.reset(new gpuSolver::MultigridGaussSeidelPreconditioner(be, h, perms, pre, post, vcycles,
                                                                 omega));
    } else if (smoother == 1) {
      pc.reset(new gpuSolver::MultigridBlockGaussSeidelPreconditioner(be, h, perms, pre, post,
                                                                      coarse, omega, vcycles));
    } else if (smoother == 2) {
      pc.reset(new gpuSolver::MultigridDampedJacobiPreconditioner(be, h, perms, pre, post, vcycles, omega));
    } else if (smoother == 3) {
      pc.reset(new gpuSolver::MultigridBlockJacobiPreconditioner(be, h, perms, pre, post, coarse, omega,
                                                                 vcycles));
    } else {
      pc.reset(new gpuSolver::MultigridHybridBlockPreconditioner(be, h, perms, pre, post, coarse, omega,
                                                                 vcycles));
    }
    gpuSolver::CGSolver solver(be, *pc, h.A[0], perms[0]);
    solver.setTolerance(tol);
    solver.setMaxIterations(max_iter);
    auto t1 = Clock::now();
    Eigen::VectorXf bv(n0), xv(n0);
    std::memcpy(bv.data(), b, sizeof(float) * n0);
    std::memcpy(xv.data(), x, sizeof(float) * n0);
    auto t2 = Clock::now();
    solver.solve(bv, xv);
    auto t3 = Clock::now();
    std::memcpy(x, xv.data(), sizeof(float) * n0);
    *iterations = static_cast<int>(solver.getNbOfIterations());
    if (setup_ms) *setup_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (solve_ms) *solve_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
  });
}

// HierarchicalReordering::compute on an AMGHierarchy given level by level
// (FP32 values): one (old_to_new, new_to_old) pair per level, finest first.
int gsref_hierarchical_reordering(int nlevels, const gsref_csr *A, const gsref_csr *P, const gsref_csr *R,
                                  int *const *old_to_new, int *const *new_to_old) {
  return guarded([&] {
    gpuSolver::AMGHierarchy h;
    for (int k = 0; k < nlevels; ++k) {
      h.A.push_back(make_matrix(A[k].rows, A[k].cols, A[k].rowptr, A[k].col, A[k].val));
      if (k + 1 < nlevels) {
        h.P.push_back(make_matrix(P[k].rows, P[k].cols, P[k].rowptr, P[k].col, P[k].val));
        h.R.push_back(make_matrix(R[k].rows, R[k].cols, R[k].rowptr, R[k].col, R[k].val));
      }
    }
    const std::vector<gpuSolver::Permutation> perms = gpuSolver::HierarchicalReordering().compute(h);
    for (int k = 0; k < nlevels; ++k) {
      std::memcpy(old_to_new[k], perms[k].oldToNew(), sizeof(int) * perms[k].size());
      std::memcpy(new_to_old[k], perms[k].newToOld(), sizeof(int) * perms[k].size());
    }
  });
}

// CGSolver with a single-level preconditioner: 0 = Identity, 1 = Jacobi,
// 2 = SymmetricGaussSeidel(omega, sweeps), 3 = DampedJacobi(sweeps, omega),
// 4 = BlockJacobi(sweeps, omega), 5 = BlockGaussSeidel(omega, sweeps).
int gsref_pcg(int n, const int *rowptr, const int *col, const float *val, const int *old_to_new,
              const int *new_to_old, int preconditioner, float omega, int sweeps, float tol,
              int max_iter, const float *b, float *x, int *iterations) {
  return guarded([&] {
    gpuSolver::CPUBackend be;
    std::unique_ptr<gpuSolver::Preconditioner> pc;
    if (preconditioner == 0) pc.reset(new gpuSolver::IdentityPreconditioner());
    else if (preconditioner == 1) pc.reset(new gpuSolver::JacobiPreconditioner());
    else if (preconditioner == 2) pc.reset(new gpuSolver::SymmetricGaussSeidelPreconditioner(omega, sweeps));
    else if (preconditioner == 3) pc.reset(new gpuSolver::DampedJacobiPreconditioner(sweeps, omega));
    else if (preconditioner == 4) pc.reset(new gpuSolver::BlockJacobiPreconditioner(sweeps, omega));
    else pc.reset(new gpuSolver::BlockGaussSeidelPreconditioner(omega, sweeps));
    SpMat A = make_matrix(n, n, rowptr, col, val);
    std::unique_ptr<gpuSolver::CGSolver> solver;
    std::unique_ptr<gpuSolver::Permutation> p;
    if (old_to_new != nullptr) {
      p.reset(new gpuSolver::Permutation(n, old_to_new, new_to_old));
      solver.reset(new gpuSolver::CGSolver(be, *pc, A, *p));
    } else {
      solver.reset(new gpuSolver::CGSolver(be, *pc, A));
    }
    solver->setTolerance(tol);
    solver->setMaxIterations(max_iter);
    Eigen::VectorXf bv(n), xv(n);
    std::memcpy(bv.data(), b, sizeof(float) * n);
    std::memcpy(xv.data(), x, sizeof(float) * n);
    solver->solve(bv, xv);
    std::memcpy(x, xv.data(), sizeof(float) * n);
    *iterations = static_cast<int>(solver->getNbOfIterations());
  });
}

}  // extern "C"
