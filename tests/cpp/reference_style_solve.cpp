// A program written the way the reference's examples drive the solver
// (examples/multigridPoisson/mainTetmeshPoisson.cc:63-98,436-597), compiled
// against include/GPUSolver and linked with libgpusolver_b200.so.
//   usage: reference_style_solve <side> <rhs.bin> <x_out.bin> [jacobi]
// With "jacobi" the CG uses a DampedJacobiPreconditioner(4, 0.9) instead of
// the multigrid one (examples/elasticity/cantileverBeam.cc:432); with
// "gpu-setup" the hierarchy is built on the GPU (buildOnDevice).
// Reads the FP32 right-hand side, writes the FP32 solution, prints
// "levels <L> iterations <k>".
#include <GPUSolver/AMGHierarchyBuilder.h>
#include <GPUSolver/CGSolver.h>
#include <GPUSolver/GraphColoring.h>
#include <GPUSolver/Preconditioners/DampedJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridGaussSeidelPreconditioner.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static gpuSolver::CsrMatrix poisson7(int m) {
  std::vector<int> rp{0}, ci;
  std::vector<double> v;
  auto id = [m](int x, int y, int z) { return (z * m + y) * m + x; };
  for (int z = 0; z < m; ++z)
    for (int y = 0; y < m; ++y)
      for (int x = 0; x < m; ++x) {
        const int i = id(x, y, z);
        auto add = [&](int j, double a) { ci.push_back(j), v.push_back(a); };
        if (z > 0) add(i - m * m, -1);
        if (y > 0) add(i - m, -1);
        if (x > 0) add(i - 1, -1);
        add(i, 6);
        if (x + 1 < m) add(i + 1, -1);
        if (y + 1 < m) add(i + m, -1);
        if (z + 1 < m) add(i + m * m, -1);
        rp.push_back(static_cast<int>(ci.size()));
      }
  return gpuSolver::CsrMatrix(m * m * m, m * m * m, rp, ci, v);
}

int main(int argc, char **argv) {
  if (argc != 4 && argc != 5) return 2;
  const bool jacobi = argc == 5 && std::string(argv[4]) == "jacobi";
  const bool gpu_setup = argc == 5 && std::string(argv[4]) == "gpu-setup";
  const int side = std::atoi(argv[1]);
  const gpuSolver::CsrMatrix K = poisson7(side);
  const int n = K.rows();
  std::vector<float> b(n), x(n, 0.0f);
  FILE *f = std::fopen(argv[2], "rb");
  if (!f || std::fread(b.data(), sizeof(float), n, f) != static_cast<size_t>(n)) return 3;
  std::fclose(f);

  gpuSolver::SmoothedAggregationCoarsener coarsener(1, 0.1f);
  gpuSolver::AMGHierarchyBuilder builder(coarsener, 10, 200);
  gpuSolver::AMGHierarchy H = gpu_setup ? builder.buildOnDevice(K, 0) : builder.build(K);
  std::vector<gpuSolver::Permutation> perms;
  gpuSolver::RCMReordering rcm;
  for (const auto &A : H.A) {
    std::vector<int> o2n(A.rows()), n2o(A.rows());
    rcm.compute(A.rows(), A.rowPtr.data(), A.colIdx.data(), o2n.data(), n2o.data());
    perms.emplace_back(A.rows(), o2n.data(), n2o.data());
  }
  gpuSolver::CudaBackend backend;
  gpuSolver::MultigridGaussSeidelPreconditioner pc(backend, H, perms, 1, 1, 1, 1.0f);
  gpuSolver::DampedJacobiPreconditioner jpc(4, 0.9f);
  gpuSolver::CGSolver solver(backend, jacobi ? static_cast<gpuSolver::Preconditioner &>(jpc) : pc, K,
                             perms[0]);
  solver.setTolerance(1e-6f);
  solver.setMaxIterations(jacobi ? 1000 : 100);
  solver.solve(b, x);

  gpuSolver::GraphColoring coloring;
  coloring.compute(n, K.rowPtr.data(), K.colIdx.data());
  std::printf("levels %zu iterations %zu colors %zu\n", H.levels(), solver.getNbOfIterations(),
              coloring.numberOfColors());
  f = std::fopen(argv[3], "wb");
  if (!f) return 4;
  std::fwrite(x.data(), sizeof(float), n, f);
  std::fclose(f);
  return 0;
}
