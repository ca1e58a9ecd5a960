// Host-side behaviour of the C++ API mirror (no GPU needed): argument
// validation and error messages (include/GPUSolver/Permutation.h:10-33,
// src/GraphColoring.cc of the reference), the hierarchy builder, RCM and the
// colouring, printed as "key value" lines for the test to compare.
#include <GPUSolver/AMGHierarchyBuilder.h>
#include <GPUSolver/CGSolver.h>
#include <GPUSolver/GraphColoring.h>
#include <GPUSolver/Preconditioners/MultigridBlockGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridGaussSeidelPreconditioner.h>
#include <GPUSolver/ReorderingStrategies/HierarchicalReordering.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>

#include <cstdio>
#include <functional>
#include <string>
#include <vector>

static gpuSolver::CsrMatrix poisson7(int m) {
  std::vector<int> rp{0}, ci;
  std::vector<double> v;
  for (int z = 0; z < m; ++z)
    for (int y = 0; y < m; ++y)
      for (int x = 0; x < m; ++x) {
        const int i = (z * m + y) * m + x;
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

static void expect_throw(const char *key, const std::function<void()> &f) {
  try {
    f();
    std::printf("%s no-throw\n", key);
  } catch (const std::runtime_error &e) {
    std::printf("%s throws: %s\n", key, e.what());
  }
}

int main() {
  using namespace gpuSolver;
  expect_throw("perm_size0", [] { Permutation p(0, nullptr, nullptr); });
  expect_throw("perm_null", [] { Permutation p(3, nullptr, nullptr); });
  const int bad_o2n[3] = {0, 1, 3}, ok_n2o[3] = {0, 1, 2};
  expect_throw("perm_range", [&] { Permutation p(3, bad_o2n, ok_n2o); });
  const int o2n[3] = {1, 2, 0}, wrong_n2o[3] = {1, 2, 0};
  expect_throw("perm_inverse", [&] { Permutation p(3, o2n, wrong_n2o); });
  expect_throw("coloring_uninit", [] { GraphColoring c; c.colors(); });
  expect_throw("builder_levels", [] { AMGHierarchyBuilder b(SmoothedAggregationCoarsener(1, 0.1f), 0, 10); });

  const CsrMatrix K = poisson7(12);
  AMGHierarchyBuilder builder(SmoothedAggregationCoarsener(1, 0.1f), 10, 50);
  AMGHierarchy H = builder.build(K);
  std::printf("null_nullspace_levels %zu\n", builder.build(K, nullptr).A.size());
  {
    const std::vector<float> modes(K.rows(), 1.0f);
    expect_throw("nullspace_modes", [&] { builder.build(K, &modes); });
  }
  std::printf("levels %zu\n", H.levels());
  for (std::size_t k = 0; k < H.levels(); ++k) std::printf("level %zu rows %d nnz %d\n", k, H.A[k].rows(), H.A[k].nonZeros());

  std::vector<Permutation> perms;
  long long sig = 0;
  for (const auto &A : H.A) {
    std::vector<int> a(A.rows()), b(A.rows());
    RCMReordering().compute(A.rows(), A.rowPtr.data(), A.colIdx.data(), a.data(), b.data());
    for (int i = 0; i < A.rows(); ++i) sig = (sig * 31 + a[i]) % 1000000007LL;
    perms.emplace_back(A.rows(), a.data(), b.data());
  }
  std::printf("rcm_signature %lld\n", sig);
  long long hsig = 0;
  for (const Permutation &p : HierarchicalReordering().compute(H))
    for (std::size_t i = 0; i < p.size(); ++i) hsig = (hsig * 31 + p.oldToNew()[i]) % 1000000007LL;
  std::printf("hierarchical_signature %lld\n", hsig);
  GraphColoring col;
  col.compute(K.rows(), K.rowPtr.data(), K.colIdx.data());
  std::printf("colors %zu offsets %zu\n", col.numberOfColors(), col.colorOffsets().size());

  // the C ABI's extensions without a GPU: the host build of the independent-set
  // aggregation, the smallest-last colouring, argument errors
  {
    gs_host_csr *m = nullptr;
    gs_host_csr_create(K.rows(), K.cols(), K.rowPtr.data(), K.colIdx.data(), K.values.data(), &m);
    gs_hierarchy *h = nullptr;
    gs_setup_stats st;
    const int rc = gs_hierarchy_build_ex(m, 1, 0.1, 10, 50, 1, -1, &st, &h);
    std::printf("mis2_rc %d levels %d", rc, rc == GS_OK ? gs_hierarchy_num_levels(h) : -1);
    for (int k = 0; rc == GS_OK && k < gs_hierarchy_num_levels(h); ++k) {
      int r = 0, c = 0, nz = 0;
      gs_hierarchy_matrix_info(h, k, 0, &r, &c, &nz);
      std::printf(" %d", r);
    }
    std::printf("\n");
    if (h != nullptr) gs_hierarchy_destroy(h);
    gs_hierarchy *h2 = nullptr;
    const int rc2 = gs_hierarchy_build_ex(m, 1, 0.1, 10, 50, 0, 0, nullptr, &h2);
    std::printf("gpu_sequential_rc %d %s\n", rc2, gs_last_error());
    gs_host_csr_destroy(m);
    std::vector<int> colors(K.rows()), verts(K.rows()), offs(K.rows() + 1);
    int nc = 0;
    gs_smallest_last_coloring(K.rows(), K.rowPtr.data(), K.colIdx.data(), colors.data(), verts.data(), offs.data(), &nc);
    std::printf("smallest_last_colors %d\n", nc);
    double t4[4];
    std::printf("setup_times_null %d\n", gs_solver_setup_times(nullptr, t4));
  }

  CudaBackend backend;
  MultigridGaussSeidelPreconditioner pc(backend, H, perms, 1, 1, 1, 1.0f);
  std::printf("coarse_steps %d smoother %d reference_vcycle %d\n", pc.options().coarse_steps,
              pc.options().smoother, pc.options().reference_vcycle);
  std::vector<Permutation> short_perms;
  short_perms.emplace_back(perms[0].size(), perms[0].oldToNew(), perms[0].newToOld());
  expect_throw("pc_perm_count", [&] { MultigridGaussSeidelPreconditioner p(backend, H, short_perms, 1, 1, 1, 1.0f); });
  expect_throw("solver_wrong_matrix", [&] { CGSolver s(backend, pc, poisson7(5)); });
  // Without a CUDA device this reports the library's error; with one it solves.
  try {
    CGSolver s(backend, pc, K);
    std::vector<double> b(K.rows(), 1.0), x(K.rows(), 0.0);
    expect_throw("solve_wrong_size", [&] { std::vector<double> y(3); s.solve(b, y); });
    s.solve(b, x);
    std::printf("device_solve iterations %zu\n", s.getNbOfIterations());
  } catch (const std::runtime_error &e) {
    std::printf("device_solve throws: %s\n", e.what());
  }
  return 0;
}
