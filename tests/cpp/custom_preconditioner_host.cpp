// CGSolver of the C++ mirror with preconditioners written by the caller
// against the reference's interface (initialize / apply), on the host test
// backend: a Jacobi preconditioner as src/Preconditioners/JacobiPreconditioner.cc
// computes it, and a symmetric Gauss-Seidel one built on the mirror's smoother.
//   usage: custom_preconditioner_host <side> <jacobi|sgs> <rcm 0|1> <b.bin> <x_out.bin>
// Poisson 7-point matrix of side^3 rows, tolerance 1e-5, at most 500 iterations;
// prints "iterations <k>".
#include <GPUSolver/CGSolver.h>
#include <GPUSolver/ReorderingStrategies/RCMReordering.h>
#include <GPUSolver/Smoothers/SymmetricGaussSeidelSmoother.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "host_backend.h"

using namespace gpuSolver;

// z = D^-1 r with D^-1 the FP32 reciprocals of the diagonal
class MyJacobi : public Preconditioner {
 public:
  void initialize(Backend &backend, const HostCSRMatrix &host, const DeviceCSRMatrix &) override {
    std::vector<float> inv(host.rows());
    for (std::size_t r = 0; r < host.rows(); ++r)
      for (int k = host.activeRowPtr()[r]; k < host.activeRowPtr()[r + 1]; ++k)
        if (host.activeColPtr()[k] == static_cast<int>(r)) inv[r] = 1.0f / host.activeValPtr()[k];
    inv_.reset(backend.createVector(inv.size(), inv.data()));
  }
  void apply(Backend &backend, BackendEncoder &encoder, const DeviceVector &input, DeviceVector &output) override {
    backend.encodeCopy(encoder, input, output);
    backend.encodeScaleVector(encoder, *inv_, output);
  }

 private:
  std::unique_ptr<DeviceVector> inv_;
};

// z = 0, then `sweeps` symmetric Gauss-Seidel steps with weight omega
class MySgs : public Preconditioner {
 public:
  MySgs(float omega, std::size_t sweeps) : smoother_(omega), sweeps_(sweeps) {}
  void initialize(Backend &backend, const HostCSRMatrix &host, const DeviceCSRMatrix &device) override {
    smoother_.initialize(backend, host, device);
  }
  void apply(Backend &backend, BackendEncoder &encoder, const DeviceVector &input, DeviceVector &output) override {
    backend.encodeSetZero(encoder, output);
    smoother_.smooth(backend, encoder, input, output, sweeps_);
  }

 private:
  SymmetricGaussSeidelSmoother smoother_;
  std::size_t sweeps_;
};

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
        add(i, 6 + 0.05 * (i % 7));
        if (x + 1 < m) add(i + 1, -1);
        if (y + 1 < m) add(i + m, -1);
        if (z + 1 < m) add(i + m * m, -1);
        rp.push_back(static_cast<int>(ci.size()));
      }
  return CsrMatrix(m * m * m, m * m * m, rp, ci, v);
}

int main(int argc, char **argv) {
  if (argc != 6) return 2;
  const CsrMatrix K = poisson7(std::atoi(argv[1]));
  const std::string kind = argv[2];
  const bool use_rcm = std::atoi(argv[3]) != 0;
  const std::size_t n = static_cast<std::size_t>(K.rows());
  std::vector<float> b(n), x(n, 0.0f);
  FILE *f = std::fopen(argv[4], "rb");
  if (!f || std::fread(b.data(), sizeof(float), n, f) != n) return 3;
  std::fclose(f);

  hostbackend::HostBackend backend;
  std::unique_ptr<Preconditioner> pc;
  if (kind == "jacobi") pc.reset(new MyJacobi);
  else pc.reset(new MySgs(1.2f, 2));
  std::unique_ptr<Permutation> perm;
  if (use_rcm) {
    std::vector<int> o2n(n), n2o(n);
    RCMReordering().compute(n, K.rowPtr.data(), K.colIdx.data(), o2n.data(), n2o.data());
    perm.reset(new Permutation(n, o2n.data(), n2o.data()));
  }
  std::unique_ptr<CGSolver> solver(perm ? new CGSolver(backend, *pc, K, *perm) : new CGSolver(backend, *pc, K));
  solver->setTolerance(1e-5f);
  solver->setMaxIterations(500);
  solver->solve(b, x);
  f = std::fopen(argv[5], "wb");
  if (!f || std::fwrite(x.data(), sizeof(float), n, f) != n) return 4;
  std::fclose(f);
  std::printf("iterations %zu custom %d\n", solver->getNbOfIterations(), pc->custom() ? 1 : 0);
  return 0;
}
