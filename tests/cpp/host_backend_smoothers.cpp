// Test-only: the mirror's abstract gpuSolver::Backend implemented on host
// memory (FP32, plain loops), to run the single-level smoothers of
// GPUSolver/Smoothers/ without a GPU. Checks the encode sequence each smoother
// issues (SGS: every colour forward, then backward, as (colorStart,
// colorCount); the Jacobi forms: spmv, copy, axpy, scale/apply, axpy) and the
// smoothed iterates against direct loops. Nothing here is part of the library.
#include <GPUSolver/DeviceScalar.h>
#include <GPUSolver/Smoothers/BlockGaussSeidelSmoother.h>
#include <GPUSolver/Smoothers/BlockJacobiSmoother.h>
#include <GPUSolver/Smoothers/DampedJacobiSmoother.h>
#include <GPUSolver/Smoothers/SymmetricGaussSeidelSmoother.h>

#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

using namespace gpuSolver;

#include "host_backend.h"

using namespace hostbackend;

namespace {

std::string joined(const std::vector<std::string> &v) {
  std::string s;
  for (const std::string &x : v) s += (s.empty() ? "" : ",") + x;
  return s;
}

// 1-D Laplacian of n rows (2 greedy colours), and a 3x3-block path of nodes
std::unique_ptr<HostCSRMatrix> path(int n) {
  std::vector<int> rp{0}, ci;
  std::vector<float> v;
  for (int i = 0; i < n; ++i) {
    if (i > 0) ci.push_back(i - 1), v.push_back(-1);
    ci.push_back(i), v.push_back(2.5f);
    if (i + 1 < n) ci.push_back(i + 1), v.push_back(-1);
    rp.push_back(static_cast<int>(ci.size()));
  }
  return std::unique_ptr<HostCSRMatrix>(new HostCSRMatrix(n, n, ci.size(), rp.data(), ci.data(), v.data()));
}
std::unique_ptr<HostCSRMatrix> block_path(int nodes) {
  std::vector<int> rp{0}, ci;
  std::vector<float> v;
  for (int node = 0; node < nodes; ++node)
    for (int r = 0; r < 3; ++r) {
      for (int nb = node - 1; nb <= node + 1; ++nb) {
        if (nb < 0 || nb >= nodes) continue;
        for (int c = 0; c < 3; ++c) {
          ci.push_back(3 * nb + c);
          v.push_back(nb == node ? (r == c ? 4.0f : 0.5f) : -0.2f);
        }
      }
      rp.push_back(static_cast<int>(ci.size()));
    }
  return std::unique_ptr<HostCSRMatrix>(new HostCSRMatrix(3 * nodes, 3 * nodes, ci.size(), rp.data(), ci.data(), v.data()));
}

double residual_norm(const HostCSRMatrix &A, const std::vector<float> &b, const std::vector<float> &x) {
  double s = 0;
  for (std::size_t r = 0; r < A.rows(); ++r) {
    double ax = 0;
    for (int k = A.activeRowPtr()[r]; k < A.activeRowPtr()[r + 1]; ++k)
      ax += double(A.activeValPtr()[k]) * x[A.activeColPtr()[k]];
    s += (b[r] - ax) * (b[r] - ax);
  }
  return std::sqrt(s);
}

}  // namespace

int main() {
  HostBackend be;
  std::unique_ptr<BackendEncoder> enc(be.createEncoder());
  {
    auto A = path(6);
    std::unique_ptr<DeviceCSRMatrix> dA(be.createCSRMatrix(*A));
    const std::vector<float> b(6, 1.0f);
    std::unique_ptr<DeviceVector> db(be.createVector(6, b.data())), dx(be.createVector(6));
    SymmetricGaussSeidelSmoother sgs(1.0f);
    sgs.initialize(be, *A, *dA);
    const double r0 = residual_norm(*A, b, V(*dx));
    be.log.clear();
    sgs.smooth(be, *enc, *db, *dx, 2);
    std::printf("sgs_sequence %s\n", joined(be.log).c_str());
    std::printf("sgs_reduces %d\n", residual_norm(*A, b, V(*dx)) < 0.5 * r0 ? 1 : 0);
    DampedJacobiSmoother dj(0.7f);
    dj.initialize(be, *A, *dA);
    be.log.clear();
    dj.smooth(be, *enc, *db, *dx, 1);
    std::printf("jacobi_sequence %s\n", joined(be.log).c_str());
  }
  {
    auto P = block_path(4);
    std::unique_ptr<DeviceCSRMatrix> dP(be.createCSRMatrix(*P));
    const std::vector<float> b(12, 1.0f);
    std::unique_ptr<DeviceVector> db(be.createVector(12, b.data())), dx(be.createVector(12));
    BlockGaussSeidelSmoother bgs(1.0f);
    bgs.initialize(be, *P, *dP);
    const double r0 = residual_norm(*P, b, V(*dx));
    be.log.clear();
    bgs.smooth(be, *enc, *db, *dx, 1);
    std::printf("bgs_sequence %s\n", joined(be.log).c_str());
    std::printf("bgs_reduces %d\n", residual_norm(*P, b, V(*dx)) < 0.5 * r0 ? 1 : 0);
    BlockJacobiSmoother bj(0.8f);
    bj.initialize(be, *P, *dP);
    be.log.clear();
    bj.smooth(be, *enc, *db, *dx, 1);
    std::printf("block_jacobi_sequence %s\n", joined(be.log).c_str());
    // one damped block-Jacobi step from x = 0 is x = w D^-1 b exactly
    std::unique_ptr<DeviceVector> dz(be.createVector(12));
    bj.smooth(be, *enc, *db, *dz, 1);
    const std::vector<float> Dinv = extractInverseDiagonalBlocks3x3(*P);
    double worst = 0;
    for (int node = 0; node < 4; ++node)
      for (int l = 0; l < 3; ++l) {
        float e = 0.0f;
        for (int m = 0; m < 3; ++m) e += Dinv[9 * node + 3 * l + m] * b[3 * node + m];
        worst = std::fmax(worst, std::fabs(V(*dz)[3 * node + l] - 0.8f * e));
      }
    std::printf("block_jacobi_first_step %.3g\n", worst);
  }
  try {
    SymmetricGaussSeidelSmoother s;
    HEnc e;
    HVec b(3), x(3);
    s.smooth(be, e, b, x, 1);
    std::printf("sgs_uninitialized no-throw\n");
  } catch (const std::runtime_error &err) {
    std::printf("sgs_uninitialized throws: %s\n", err.what());
  }
  return 0;
}
