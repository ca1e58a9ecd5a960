// The kernel-level Backend of the C++ API mirror (GPUSolver/cuda/CudaBackend.h)
// used the way the reference's CUDA tests use theirs: the known answers of
// tests/cuda/testCudaGaussSeidel.cc, testCudaSpmv.cc, testCudaBlockOps.cc,
// testCudaVectorOps.cc and testCudaScalarOps.cc, then the four single-level
// smoothers against plain FP32 loops on the host (the reference's GPU-vs-CPU
// smoother tolerance, 1e-5). Without a CUDA device it prints the error the
// first device object raises.
#include <GPUSolver/HostELLMatrix.h>
#include <GPUSolver/Smoothers/BlockGaussSeidelSmoother.h>
#include <GPUSolver/Smoothers/BlockJacobiSmoother.h>
#include <GPUSolver/Smoothers/DampedJacobiSmoother.h>
#include <GPUSolver/Smoothers/SymmetricGaussSeidelSmoother.h>
#include <GPUSolver/cuda/CudaBackend.h>

#include <cmath>
#include <cstdio>
#include <functional>
#include <memory>
#include <string>
#include <vector>

using namespace gpuSolver;

struct Trip {
  int r, c;
  float v;
};

static std::unique_ptr<HostCSRMatrix> host_csr(int n, const std::vector<Trip> &t) {
  std::vector<int> rp(n + 1, 0), ci;
  std::vector<float> v;
  for (int r = 0; r < n; ++r) {
    for (const Trip &e : t)
      if (e.r == r) ci.push_back(e.c), v.push_back(e.v);
    rp[r + 1] = static_cast<int>(ci.size());
  }
  return std::unique_ptr<HostCSRMatrix>(new HostCSRMatrix(n, n, ci.size(), rp.data(), ci.data(), v.data()));
}

static std::string join(const float *p, std::size_t n) {
  std::string s;
  for (std::size_t i = 0; i < n; ++i) {
    char b[32];
    std::snprintf(b, sizeof b, "%s%g", i ? " " : "", static_cast<double>(p[i]));
    s += b;
  }
  return s;
}

static void expect_throw(const char *key, const std::function<void()> &f) {
  try {
    f();
    std::printf("%s no-throw\n", key);
  } catch (const std::runtime_error &e) {
    std::printf("%s throws: %s\n", key, e.what());
  }
}

// 2-D 5-point Laplacian on an m x m grid, diagonal 4 + small row-dependent shift
static std::unique_ptr<HostCSRMatrix> laplace2d(int m) {
  std::vector<Trip> t;
  for (int y = 0; y < m; ++y)
    for (int x = 0; x < m; ++x) {
      const int i = y * m + x;
      if (y > 0) t.push_back({i, i - m, -1});
      if (x > 0) t.push_back({i, i - 1, -1});
      t.push_back({i, i, 4.0f + 0.01f * static_cast<float>(i % 5)});
      if (x + 1 < m) t.push_back({i, i + 1, -1});
      if (y + 1 < m) t.push_back({i, i + m, -1});
    }
  return host_csr(m * m, t);
}

// 3x3 blocks along a path of nodes, SPD diagonal blocks
static std::unique_ptr<HostCSRMatrix> block_path(int nodes) {
  std::vector<Trip> t;
  for (int node = 0; node < nodes; ++node)
    for (int r = 0; r < 3; ++r)
      for (int nb = node - 1; nb <= node + 1; ++nb) {
        if (nb < 0 || nb >= nodes) continue;
        for (int c = 0; c < 3; ++c)
          t.push_back({3 * node + r, 3 * nb + c, nb == node ? (r == c ? 4.0f + 0.5f * node : 0.5f) : -0.2f});
      }
  return host_csr(3 * nodes, t);
}

static double rel_diff(const float *a, const std::vector<float> &b) {
  double num = 0, den = 0;
  for (std::size_t i = 0; i < b.size(); ++i) {
    num += (double(a[i]) - b[i]) * (double(a[i]) - b[i]);
    den += double(b[i]) * b[i];
  }
  return std::sqrt(num / den);
}

int main() {
  CudaBackend backend;
  try {
    std::unique_ptr<DeviceVector> probe(backend.createVector(4));
  } catch (const std::runtime_error &e) {
    std::printf("no_device %s\n", e.what());
    return 0;
  }
  std::unique_ptr<BackendEncoder> enc(backend.createEncoder());

  // ---- testCudaGaussSeidel.cc: 4x4 tridiagonal, colours {0, 2} then {1, 3} ----
  auto T = host_csr(4, {{0, 0, 4}, {0, 1, -1}, {1, 0, -1}, {1, 1, 4}, {1, 2, -1}, {2, 1, -1}, {2, 2, 4}, {2, 3, -1},
                        {3, 2, -1}, {3, 3, 4}});
  std::unique_ptr<DeviceCSRMatrix> A(backend.createCSRMatrix(*T));
  const int order[4] = {0, 2, 1, 3};
  const float rhs4[4] = {4, 8, 12, 16};
  std::unique_ptr<DeviceIndexVector> cv(backend.createIndexVector(4, order));
  std::unique_ptr<DeviceVector> b(backend.createVector(4, rhs4)), x(backend.createVector(4));
  backend.encodeGaussSeidelColor(*enc, *A, *cv, 0, 2, *b, *x, 1.0f);
  backend.submitAndWait(*enc);
  std::printf("gs_color0 %s\n", join(x->download(), 4).c_str());
  backend.encodeGaussSeidelColor(*enc, *A, *cv, 2, 2, *b, *x, 1.0f);
  backend.submitAndWait(*enc);
  std::printf("gs_sweep %s\n", join(x->download(), 4).c_str());
  expect_throw("gs_range", [&] { backend.encodeGaussSeidelColor(*enc, *A, *cv, 3, 2, *b, *x, 1.0f); });

  // ---- testCudaSpmv.cc: y = A x, values updated in place; dot ----
  auto S3 = host_csr(3, {{0, 0, 4}, {0, 1, 1}, {1, 0, 1}, {1, 1, 3}, {1, 2, 2}, {2, 1, 2}, {2, 2, 5}});
  std::unique_ptr<DeviceCSRMatrix> A3(backend.createCSRMatrix(*S3));
  const float x3[3] = {1, 2, 3}, y3[3] = {4, 5, 6};
  std::unique_ptr<DeviceVector> vx(backend.createVector(3, x3)), vy(backend.createVector(3));
  backend.spmv(*A3, *vx, *vy);
  std::printf("spmv %s\n", join(vy->download(), 3).c_str());
  auto S2 = host_csr(2, {{0, 0, 2}, {0, 1, 1}, {1, 0, 1}, {1, 1, 3}});
  std::unique_ptr<DeviceCSRMatrix> A2(backend.createCSRMatrix(*S2));
  const float nv[4] = {4, 2, 2, 6}, x2[2] = {1, 2};
  A2->updateValues(nv, 4);
  std::unique_ptr<DeviceVector> wx(backend.createVector(2, x2)), wy(backend.createVector(2));
  backend.spmv(*A2, *wx, *wy);
  std::printf("spmv_updated %s\n", join(wy->download(), 2).c_str());
  expect_throw("spmv_shape", [&] { backend.spmv(*A3, *wx, *wy); });
  expect_throw("update_count", [&] { A2->updateValues(nv, 3); });
  std::unique_ptr<DeviceVector> vy3(backend.createVector(3, y3));
  std::unique_ptr<DeviceScalar> d(backend.createScalar());
  backend.encodeDot(*enc, *vx, *vy3, *d);
  backend.submitAndWait(*enc);
  std::printf("dot %g\n", static_cast<double>(d->download()));

  // ---- testCudaBlockOps.cc: c = D^-1 r ----
  const float dinv[18] = {2, 0, 0, 0, 3, 0, 0, 0, 4, 1, 1, 0, 0, 2, 0, 0, 0, 3};
  const float r6[6] = {1, 2, 3, 4, 5, 6};
  std::unique_ptr<DeviceVector> vd(backend.createVector(18, dinv)), vr(backend.createVector(6, r6)),
      vc(backend.createVector(6));
  backend.encodeApplyBlockInverses3x3(*enc, *vd, *vr, *vc);
  backend.submitAndWait(*enc);
  std::printf("block_apply %s\n", join(vc->download(), 6).c_str());

  // ---- testCudaVectorOps.cc / testCudaScalarOps.cc ----
  const float ten[3] = {10, 20, 30};
  std::unique_ptr<DeviceVector> y(backend.createVector(3, ten));
  std::unique_ptr<DeviceScalar> three(backend.createScalar(3.0f));
  backend.axpy(2.0f, *vx, *y);
  backend.scale(*y, 0.5f);
  std::printf("axpy_scale %s\n", join(y->download(), 3).c_str());
  backend.axpy(*three, *vx, *y);
  backend.scaleVectorByVector(*vx, *y);
  std::printf("axpy_dev_scale_vector %s\n", join(y->download(), 3).c_str());
  backend.encodeCopy(*enc, *vx, *y);
  backend.submitAndWait(*enc);
  std::printf("copy %s\n", join(y->download(), 3).c_str());
  backend.encodeSetZero(*enc, *y);
  backend.submitAndWait(*enc);
  std::printf("set_zero %s\n", join(y->download(), 3).c_str());
  y->updateValues(ten, 2);  // a new size reallocates
  std::printf("resized %zu %s\n", y->size(), join(y->download(), 2).c_str());
  std::unique_ptr<DeviceScalar> s6(backend.createScalar(6.0f)), s4(backend.createScalar(4.0f)), o(backend.createScalar());
  backend.scalarDivide(*s6, *s4, *o);
  const double q = o->download();
  backend.scalarMultiply(*o, *s4, *o);
  backend.scalarNegate(*o, *o);
  const double neg = o->download();
  backend.scalarSet(16.0f, *o);
  backend.scalarSqrt(*o, *o);
  backend.scalarCopy(*o, *s6);
  std::printf("scalars %g %g %g\n", q, neg, static_cast<double>(s6->download()));

  // ---- smoothers against FP32 host loops ----
  {
    auto L = laplace2d(8);
    const std::size_t n = L->rows();
    std::unique_ptr<DeviceCSRMatrix> dA(backend.createCSRMatrix(*L));
    std::vector<float> bh(n), x0(n);
    for (std::size_t i = 0; i < n; ++i) bh[i] = std::sin(0.3f * i), x0[i] = 0.1f * std::cos(0.7f * i);
    const int *rp = L->activeRowPtr(), *ci = L->activeColPtr();
    const float *av = L->activeValPtr();
    auto gs_row = [&](std::vector<float> &xx, int i, float w) {
      float sum = 0, dd = 1;
      for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i) dd = av[k];
        else sum += av[k] * xx[ci[k]];
      xx[i] = (1 - w) * xx[i] + w * (bh[i] - sum) / dd;
    };
    // SGS, 2 steps, omega 1.2
    SymmetricGaussSeidelSmoother sgs(1.2f);
    sgs.initialize(backend, *L, *dA);
    std::unique_ptr<DeviceVector> db(backend.createVector(n, bh.data())), dx(backend.createVector(n, x0.data()));
    sgs.smooth(backend, *enc, *db, *dx, 2);
    backend.submitAndWait(*enc);
    GraphColoring col;
    col.compute(n, rp, ci);
    std::vector<float> xs = x0;
    const std::vector<int> &off = col.colorOffsets(), &vv = col.colorVertices();
    for (int it = 0; it < 2; ++it) {
      for (std::size_t c = 0; c + 1 < off.size(); ++c)
        for (int t = off[c]; t < off[c + 1]; ++t) gs_row(xs, vv[t], 1.2f);
      for (std::size_t c = off.size() - 1; c > 0; --c)
        for (int t = off[c - 1]; t < off[c]; ++t) gs_row(xs, vv[t], 1.2f);
    }
    std::printf("sgs_smoother %.3g colours %zu\n", rel_diff(dx->download(), xs), off.size() - 1);
    // damped Jacobi, 3 steps, omega 0.7
    DampedJacobiSmoother dj(0.7f);
    dj.initialize(backend, *L, *dA);
    dx->updateValues(x0.data(), n);
    dj.smooth(backend, *enc, *db, *dx, 3);
    backend.submitAndWait(*enc);
    std::vector<float> xj = x0, t(n);
    for (int it = 0; it < 3; ++it) {
      for (std::size_t i = 0; i < n; ++i) {
        float ax = 0, dd = 1;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
          ax += av[k] * xj[ci[k]];
          if (ci[k] == static_cast<int>(i)) dd = av[k];
        }
        t[i] = (bh[i] - ax) / dd;
      }
      for (std::size_t i = 0; i < n; ++i) xj[i] += 0.7f * t[i];
    }
    std::printf("jacobi_smoother %.3g\n", rel_diff(dx->download(), xj));
    expect_throw("sgs_omega", [] { SymmetricGaussSeidelSmoother bad(2.0f); });
    expect_throw("sgs_twice", [&] { sgs.initialize(backend, *L, *dA); });
  }
  {
    auto P = block_path(6);
    const std::size_t n = P->rows();
    std::unique_ptr<DeviceCSRMatrix> dP(backend.createCSRMatrix(*P));
    std::vector<float> bh(n), x0(n);
    for (std::size_t i = 0; i < n; ++i) bh[i] = 1.0f + 0.1f * i, x0[i] = 0.05f * i;
    const int *rp = P->activeRowPtr(), *ci = P->activeColPtr();
    const float *av = P->activeValPtr();
    const std::vector<float> Dinv = extractInverseDiagonalBlocks3x3(*P);
    auto block_update = [&](std::vector<float> &xx, const std::vector<float> &src, int node, float w) {
      float res[3];
      for (int l = 0; l < 3; ++l) {
        const int r = 3 * node + l;
        float s = 0;
        for (int k = rp[r]; k < rp[r + 1]; ++k)
          if (ci[k] / 3 != node) s += av[k] * src[ci[k]];
        res[l] = bh[r] - s;
      }
      for (int l = 0; l < 3; ++l) {
        float nvv = 0;
        for (int c = 0; c < 3; ++c) nvv += Dinv[9 * node + 3 * l + c] * res[c];
        xx[3 * node + l] = (1 - w) * xx[3 * node + l] + w * nvv;
      }
    };
    BlockGaussSeidelSmoother bgs(0.9f);
    bgs.initialize(backend, *P, *dP);
    std::unique_ptr<DeviceVector> db(backend.createVector(n, bh.data())), dx(backend.createVector(n, x0.data()));
    bgs.smooth(backend, *enc, *db, *dx, 2);
    backend.submitAndWait(*enc);
    const BlockGraph g = buildBlockGraph(*P, 3);
    GraphColoring col;
    col.compute(g.rowPtr.size() - 1, g.rowPtr.data(), g.colPtr.data());
    const std::vector<int> &off = col.colorOffsets(), &vv = col.colorVertices();
    std::vector<float> xs = x0;
    for (int it = 0; it < 2; ++it) {
      for (std::size_t c = 0; c + 1 < off.size(); ++c)
        for (int t = off[c]; t < off[c + 1]; ++t) block_update(xs, xs, vv[t], 0.9f);
      for (std::size_t c = off.size() - 1; c > 0; --c)
        for (int t = off[c - 1]; t < off[c]; ++t) block_update(xs, xs, vv[t], 0.9f);
    }
    std::printf("block_gs_smoother %.3g colours %zu\n", rel_diff(dx->download(), xs), off.size() - 1);
    BlockJacobiSmoother bj(0.6f);
    bj.initialize(backend, *P, *dP);
    dx->updateValues(x0.data(), n);
    bj.smooth(backend, *enc, *db, *dx, 3);
    backend.submitAndWait(*enc);
    // x += w D^-1 (b - A x): the block form of the update with the diagonal
    // block kept in the residual
    std::vector<float> xj = x0;
    for (int it = 0; it < 3; ++it) {
      std::vector<float> r(n);
      for (std::size_t i = 0; i < n; ++i) {
        float ax = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) ax += av[k] * xj[ci[k]];
        r[i] = bh[i] - ax;
      }
      for (std::size_t node = 0; node < n / 3; ++node)
        for (int l = 0; l < 3; ++l) {
          float c = 0;
          for (int m = 0; m < 3; ++m) c += Dinv[9 * node + 3 * l + m] * r[3 * node + m];
          xj[3 * node + l] += 0.6f * c;
        }
    }
    std::printf("block_jacobi_smoother %.3g\n", rel_diff(dx->download(), xj));
    HostELLMatrix E(*P, 4);
    std::unique_ptr<DeviceELLMatrix> dE(backend.createELLMatrix(E));
    std::printf("ell %zu %zu %zu %zu\n", dE->rows(), dE->cols(), dE->ellWidth(), dE->overflowNnz());
  }
  return 0;
}
