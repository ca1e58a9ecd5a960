// Preconditioner::initialize / apply of the C++ API mirror on the host test
// backend, the way the reference's CGSolver drives a preconditioner
// (src/CGSolver.cc:170-200): initialize with the host and device matrix,
// then apply(r, z).
//   usage: preconditioner_apply_host single <side> <omega> <sweeps> <r.bin> <out_prefix>
//            writes <out_prefix>{sgs,jacobi,damped,identity}.bin for the 7-point
//            Poisson matrix of side^3 rows (FP32 values, natural order)
//          preconditioner_apply_host multigrid <side> <r.bin> <z.bin>
//            MultigridGaussSeidelPreconditioner(1, 1, 1 V-cycle, omega 1) over the
//            builder's hierarchy with per-level RCM; r, z in the level-0 permuted order
#include <GPUSolver/AMGHierarchyBuilder.h>
#include <GPUSolver/Preconditioners/DampedJacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/IdentityPreconditioner.h>
#include <GPUSolver/Preconditioners/JacobiPreconditioner.h>
#include <GPUSolver/Preconditioners/MultigridGaussSeidelPreconditioner.h>
#include <GPUSolver/Preconditioners/SymmetricGaussSeidelPreconditioner.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <GPUSolver/SparseMatrixUtils.h>

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

static bool read(const char *path, std::vector<float> &v) {
  FILE *f = std::fopen(path, "rb");
  const bool ok = f && std::fread(v.data(), sizeof(float), v.size(), f) == v.size();
  if (f) std::fclose(f);
  return ok;
}
static bool write(const std::string &path, const float *p, std::size_t n) {
  FILE *f = std::fopen(path.c_str(), "wb");
  const bool ok = f && std::fwrite(p, sizeof(float), n, f) == n;
  if (f) std::fclose(f);
  return ok;
}

static bool run(Preconditioner &pc, hostbackend::HostBackend &be, const HostCSRMatrix &host,
                const DeviceCSRMatrix &dev, const std::vector<float> &r, const std::string &out) {
  pc.initialize(be, host, dev);
  std::unique_ptr<BackendEncoder> enc(be.createEncoder());
  std::unique_ptr<DeviceVector> dr(be.createVector(r.size(), r.data())), dz(be.createVector(r.size()));
  const std::vector<float> junk(r.size(), 7.0f);
  dz->updateValues(junk.data(), junk.size());  // apply must overwrite what was there
  pc.apply(be, *enc, *dr, *dz);
  be.submitAndWait(*enc);
  return write(out, dz->download(), r.size());
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const std::string mode = argv[1];
  hostbackend::HostBackend be;
  if (mode == "single" && argc == 7) {
    const CsrMatrix K = poisson7(std::atoi(argv[2]));
    const float omega = static_cast<float>(std::atof(argv[3]));
    const std::size_t sweeps = static_cast<std::size_t>(std::atoi(argv[4]));
    std::vector<float> r(K.rows());
    if (!read(argv[5], r)) return 3;
    const std::string out = argv[6];
    const HostCSRMatrix host(K);
    std::unique_ptr<DeviceCSRMatrix> dev(be.createCSRMatrix(host));
    SymmetricGaussSeidelPreconditioner sgs(omega, sweeps);
    JacobiPreconditioner jac;
    DampedJacobiPreconditioner damped(sweeps, omega);
    IdentityPreconditioner id;
    bool ok = run(sgs, be, host, *dev, r, out + "sgs.bin") && run(jac, be, host, *dev, r, out + "jacobi.bin") &&
              run(damped, be, host, *dev, r, out + "damped.bin") && run(id, be, host, *dev, r, out + "identity.bin");
    return ok ? 0 : 4;
  }
  if (mode == "multigrid" && argc == 5) {
    const CsrMatrix K = poisson7(std::atoi(argv[2]));
    std::vector<float> r(K.rows());
    if (!read(argv[3], r)) return 3;
    AMGHierarchyBuilder builder(SmoothedAggregationCoarsener(1, 0.1f), 10, 50);
    const AMGHierarchy H = builder.build(K);
    std::vector<Permutation> perms;
    RCMReordering rcm;
    for (const auto &A : H.A) {
      std::vector<int> o2n(A.rows()), n2o(A.rows());
      rcm.compute(A.rows(), A.rowPtr.data(), A.colIdx.data(), o2n.data(), n2o.data());
      perms.emplace_back(A.rows(), o2n.data(), n2o.data());
    }
    MultigridGaussSeidelPreconditioner pc(be, H, perms, 1, 1, 1, 1.0f);
    const HostCSRMatrix host(permuteMatrix(H.A[0], perms[0].oldToNew(), perms[0].oldToNew()));
    std::unique_ptr<DeviceCSRMatrix> dev(be.createCSRMatrix(host));
    return run(pc, be, host, *dev, r, argv[4]) ? 0 : 4;
  }
  return 2;
}
