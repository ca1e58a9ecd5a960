// The mirror's MultigridSmoother family on the host test backend: builds the
// smoothed-aggregation hierarchy of a 7-point Poisson matrix with
// AMGHierarchyBuilder, one RCM permutation per level, and applies one
// V-cycle from z = 0 to r (the reference's Multigrid*Preconditioner::apply,
// src/Preconditioners/MultigridGaussSeidelPreconditioner.cc:39-54).
//   usage: multigrid_smoother_host <side> <sgs|jacobi> <r.bin> <z_out.bin>
// r and z are FP32 in the level-0 permuted order. Prints "levels <L>" and
// the encode counts.
#include <GPUSolver/AMGHierarchyBuilder.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <GPUSolver/Smoothers/MultigridDampedJacobiSmoother.h>
#include <GPUSolver/Smoothers/MultigridGaussSeidelSmoother.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "host_backend.h"

using namespace gpuSolver;

static CsrMatrix poisson7(int m) {
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
  return CsrMatrix(m * m * m, m * m * m, rp, ci, v);
}

int main(int argc, char **argv) {
  if (argc != 5) return 2;
  const int side = std::atoi(argv[1]);
  const std::string type = argv[2];
  const CsrMatrix K = poisson7(side);
  const int n = K.rows();
  std::vector<float> r(n);
  FILE *f = std::fopen(argv[3], "rb");
  if (!f || std::fread(r.data(), sizeof(float), n, f) != static_cast<size_t>(n)) return 3;
  std::fclose(f);

  AMGHierarchyBuilder builder(SmoothedAggregationCoarsener(1, 0.1f), 10, 50);
  const AMGHierarchy H = builder.build(K);
  std::vector<Permutation> perms;
  RCMReordering rcm;
  for (const auto &A : H.A) {
    std::vector<int> o2n(A.rows()), n2o(A.rows());
    rcm.compute(A.rows(), A.rowPtr.data(), A.colIdx.data(), o2n.data(), n2o.data());
    perms.emplace_back(A.rows(), o2n.data(), n2o.data());
  }

  hostbackend::HostBackend be;
  std::unique_ptr<MultigridSmoother> mg;
  if (type == "sgs")
    mg.reset(new MultigridGaussSeidelSmoother(be, H, perms, 1, 1, 2, 1.0f));
  else
    mg.reset(new MultigridDampedJacobiSmoother(be, H, perms, 2, 2, 4, 0.7f));
  std::unique_ptr<BackendEncoder> enc(be.createEncoder());
  std::unique_ptr<DeviceVector> dr(be.createVector(n, r.data())), dz(be.createVector(n));
  be.log.clear();
  be.encodeSetZero(*enc, *dz);
  mg->smooth(be, *enc, *dr, *dz, 1);
  be.submitAndWait(*enc);
  std::size_t spmv = 0, gs = 0;
  for (const std::string &op : be.log) spmv += op == "spmv", gs += op.rfind("gs ", 0) == 0;
  f = std::fopen(argv[4], "wb");
  if (!f || std::fwrite(dz->download(), sizeof(float), n, f) != static_cast<size_t>(n)) return 4;
  std::fclose(f);
  std::printf("levels %zu spmv %zu gs %zu\n", H.A.size(), spmv, gs);
  return 0;
}
