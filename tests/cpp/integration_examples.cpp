// The two C++ examples a reader of the integration guide copies: the
// reference's AMG-PCG call sequence (examples/multigridPoisson/
// mainTetmeshPoisson.cc:436-597) on the C++ mirror, and a caller-written
// preconditioner driven by CGSolver. Compiled (syntax only) by
// tests/test_cpp_api.py against include/ so the guide's code stays valid.
#include <GPUSolver/AMGHierarchyBuilder.h>
#include <GPUSolver/CGSolver.h>
#include <GPUSolver/Preconditioners/MultigridGaussSeidelPreconditioner.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <memory>
#include <vector>

// --- example 2: a preconditioner written against the reference's interface
struct MyJacobi : gpuSolver::Preconditioner {
  std::unique_ptr<gpuSolver::DeviceVector> inv;
  void initialize(gpuSolver::Backend &be, const gpuSolver::HostCSRMatrix &A, const gpuSolver::DeviceCSRMatrix &) override {
    std::vector<float> d(A.rows());
    for (std::size_t r = 0; r < A.rows(); ++r)
      for (int k = A.activeRowPtr()[r]; k < A.activeRowPtr()[r + 1]; ++k)
        if (A.activeColPtr()[k] == int(r)) d[r] = 1.0f / A.activeValPtr()[k];
    inv.reset(be.createVector(d.size(), d.data()));
  }
  void apply(gpuSolver::Backend &be, gpuSolver::BackendEncoder &e, const gpuSolver::DeviceVector &r,
             gpuSolver::DeviceVector &z) override {
    be.encodeCopy(e, r, z);
    be.encodeScaleVector(e, *inv, z);
  }
};

void example(const gpuSolver::CsrMatrix &K, std::vector<float> &b, std::vector<float> &x) {
  // --- example 1: the reference's call sequence
  gpuSolver::SmoothedAggregationCoarsener coarsener(1, 0.1f);
  gpuSolver::AMGHierarchyBuilder builder(coarsener, 10, 1000);
  gpuSolver::AMGHierarchy H = builder.build(K);
  std::vector<gpuSolver::Permutation> perms;  // per-level RCMReordering, as buildRCMPermutationsForHierarchy
  gpuSolver::CudaBackend backend;             // = B200Backend(device 0)
  gpuSolver::MultigridGaussSeidelPreconditioner pc(backend, H, perms, 1, 1, 1, 1.0f);
  gpuSolver::CGSolver solver(backend, pc, K, perms[0]);
  solver.setTolerance(1e-6f);
  solver.solve(b, x);
  std::size_t its = solver.getNbOfIterations();
  (void)its;

  // example 2, used
  MyJacobi mine;
  gpuSolver::CGSolver custom_solver(backend, mine, K);  // same results as CGSolver + JacobiPreconditioner
}

int main() { return 0; }
