// Test-only: the mirror's abstract gpuSolver::Backend implemented on host
// memory (FP32, plain sequential loops), so that the smoother classes of
// GPUSolver/Smoothers/ run without a GPU. Every encode* call is also recorded
// by name in `log`. Nothing here is part of the library.
#pragma once
#include <GPUSolver/Backend.h>
#include <GPUSolver/BackendEncoder.h>
#include <GPUSolver/DeviceIndexVector.h>
#include <GPUSolver/DeviceScalar.h>
#include <GPUSolver/DeviceSparseMatrix.h>
#include <GPUSolver/DeviceVector.h>
#include <GPUSolver/HostSparseMatrix.h>

#include <cmath>
#include <string>
#include <vector>

namespace hostbackend {

using namespace gpuSolver;

struct HVec : DeviceVector {
  explicit HVec(std::size_t n) : v(n, 0.0f) {}
  std::size_t size() const override { return v.size(); }
  void updateValues(const float *p, std::size_t n) override { v.assign(p, p + n); }
  float *download() const override { return const_cast<float *>(v.data()); }
  std::vector<float> v;
};
struct HIdx : DeviceIndexVector {
  explicit HIdx(std::size_t n) : v(n, 0) {}
  std::size_t size() const override { return v.size(); }
  void updateValues(const int *p, std::size_t n) override { v.assign(p, p + n); }
  int *download() const override { return const_cast<int *>(v.data()); }
  std::vector<int> v;
};
struct HScalar : DeviceScalar {
  explicit HScalar(float x) : v(x) {}
  float download() const override { return v; }
  float v;
};
struct HCsr : DeviceCSRMatrix {
  explicit HCsr(const HostCSRMatrix &m)
      : n(m.rows()), c(m.cols()), rp(m.activeRowPtr(), m.activeRowPtr() + m.rows() + 1),
        ci(m.activeColPtr(), m.activeColPtr() + m.nnz()), v(m.activeValPtr(), m.activeValPtr() + m.nnz()) {}
  std::size_t rows() const override { return n; }
  std::size_t cols() const override { return c; }
  std::size_t nnz() const override { return ci.size(); }
  void updateValues(const float *p, std::size_t k) override { v.assign(p, p + k); }
  std::size_t n, c;
  std::vector<int> rp, ci;
  std::vector<float> v;
};
struct HEnc : BackendEncoder {};

inline std::vector<float> &V(const DeviceVector &x) { return const_cast<HVec &>(dynamic_cast<const HVec &>(x)).v; }
inline const std::vector<int> &I(const DeviceIndexVector &x) { return dynamic_cast<const HIdx &>(x).v; }
inline float &S(const DeviceScalar &x) { return const_cast<HScalar &>(dynamic_cast<const HScalar &>(x)).v; }
inline const HCsr &M(const DeviceCSRMatrix &x) { return dynamic_cast<const HCsr &>(x); }

class HostBackend : public Backend {
 public:
  std::vector<std::string> log;

  BackendEncoder *createEncoder() override { return new HEnc; }
  void submit(BackendEncoder &) override {}
  void submitAndWait(BackendEncoder &) override {}
  DeviceVector *createVector(std::size_t n) override { return new HVec(n); }
  DeviceVector *createVector(std::size_t n, const float *p) override {
    HVec *v = new HVec(n);
    v->updateValues(p, n);
    return v;
  }
  DeviceIndexVector *createIndexVector(std::size_t n) override { return new HIdx(n); }
  DeviceIndexVector *createIndexVector(std::size_t n, const int *p) override {
    HIdx *v = new HIdx(n);
    v->updateValues(p, n);
    return v;
  }
  DeviceScalar *createScalar() override { return new HScalar(0.0f); }
  DeviceScalar *createScalar(float x) override { return new HScalar(x); }
  DeviceCSRMatrix *createCSRMatrix(const HostCSRMatrix &m) override { return new HCsr(m); }
  DeviceELLMatrix *createELLMatrix(const HostELLMatrix &) override { throw std::runtime_error("not used"); }

  void encodeScale(BackendEncoder &, DeviceVector &x, float a) override {
    log.push_back("scale");
    for (float &e : V(x)) e *= a;
  }
  void encodeScale(BackendEncoder &e, DeviceVector &x, const DeviceScalar &a) override { encodeScale(e, x, S(a)); }
  void encodeCopy(BackendEncoder &, const DeviceVector &x, DeviceVector &y) override {
    log.push_back("copy");
    V(y) = V(x);
  }
  void encodeScaleVector(BackendEncoder &, const DeviceVector &s, DeviceVector &y) override {
    log.push_back("scale_vector");
    for (std::size_t i = 0; i < V(y).size(); ++i) V(y)[i] *= V(s)[i];
  }
  void encodeSetZero(BackendEncoder &, DeviceVector &x) override {
    log.push_back("set_zero");
    for (float &e : V(x)) e = 0.0f;
  }
  void encodeAxpy(BackendEncoder &, float a, const DeviceVector &x, DeviceVector &y) override {
    log.push_back("axpy");
    for (std::size_t i = 0; i < V(y).size(); ++i) V(y)[i] += a * V(x)[i];
  }
  void encodeAxpy(BackendEncoder &e, const DeviceScalar &a, const DeviceVector &x, DeviceVector &y) override {
    encodeAxpy(e, S(a), x, y);
  }
  void encodeSpmv(BackendEncoder &, const DeviceCSRMatrix &A, const DeviceVector &x, DeviceVector &y) override {
    log.push_back("spmv");
    const HCsr &m = M(A);
    for (std::size_t r = 0; r < m.n; ++r) {
      float s = 0.0f;
      for (int k = m.rp[r]; k < m.rp[r + 1]; ++k) s += m.v[k] * V(x)[m.ci[k]];
      V(y)[r] = s;
    }
  }
  void encodeGaussSeidelColor(BackendEncoder &, const DeviceCSRMatrix &A, const DeviceIndexVector &cv,
                              std::size_t start, std::size_t count, const DeviceVector &b, DeviceVector &x,
                              float w) override {
    log.push_back("gs " + std::to_string(start) + " " + std::to_string(count));
    const HCsr &m = M(A);
    for (std::size_t t = start; t < start + count; ++t) {
      const int i = I(cv)[t];
      float s = 0.0f, d = 1.0f;
      for (int k = m.rp[i]; k < m.rp[i + 1]; ++k)
        if (m.ci[k] == i) d = m.v[k];
        else s += m.v[k] * V(x)[m.ci[k]];
      V(x)[i] = (1 - w) * V(x)[i] + w * (V(b)[i] - s) / d;
    }
  }
  void encodeDot(BackendEncoder &, const DeviceVector &x, const DeviceVector &y, DeviceScalar &r) override {
    float s = 0.0f;
    for (std::size_t i = 0; i < V(x).size(); ++i) s += V(x)[i] * V(y)[i];
    S(r) = s;
  }
  void encodeScalarDivide(BackendEncoder &, const DeviceScalar &a, const DeviceScalar &b, DeviceScalar &o) override {
    S(o) = S(a) / S(b);
  }
  void encodeScalarMultiply(BackendEncoder &, const DeviceScalar &a, const DeviceScalar &b,
                            DeviceScalar &o) override {
    S(o) = S(a) * S(b);
  }
  void encodeScalarSet(BackendEncoder &, float x, DeviceScalar &o) override { S(o) = x; }
  void encodeScalarCopy(BackendEncoder &, const DeviceScalar &a, DeviceScalar &o) override { S(o) = S(a); }
  void encodeScalarNegate(BackendEncoder &, const DeviceScalar &a, DeviceScalar &o) override { S(o) = -S(a); }
  void encodeScalarSqrt(BackendEncoder &, const DeviceScalar &a, DeviceScalar &o) override { S(o) = std::sqrt(S(a)); }
  void encodeApplyBlockInverses3x3(BackendEncoder &, const DeviceVector &d, const DeviceVector &r,
                                   DeviceVector &c) override {
    log.push_back("block_apply");
    for (std::size_t node = 0; node < V(r).size() / 3; ++node)
      for (int l = 0; l < 3; ++l) {
        float s = 0.0f;
        for (int m = 0; m < 3; ++m) s += V(d)[9 * node + 3 * l + m] * V(r)[3 * node + m];
        V(c)[3 * node + l] = s;
      }
  }
  void encodeBlockGaussSeidelColor3x3(BackendEncoder &, const DeviceCSRMatrix &A, const DeviceIndexVector &cb,
                                      const DeviceVector &dinv, std::size_t begin, std::size_t count,
                                      const DeviceVector &b, DeviceVector &x, float w) override {
    log.push_back("bgs " + std::to_string(begin) + " " + std::to_string(count));
    const HCsr &m = M(A);
    for (std::size_t t = begin; t < begin + count; ++t) {
      const int node = I(cb)[t];
      float res[3];
      for (int l = 0; l < 3; ++l) {
        const int r = 3 * node + l;
        float s = 0.0f;
        for (int k = m.rp[r]; k < m.rp[r + 1]; ++k)
          if (m.ci[k] / 3 != node) s += m.v[k] * V(x)[m.ci[k]];
        res[l] = V(b)[r] - s;
      }
      for (int l = 0; l < 3; ++l) {
        float nv = 0.0f;
        for (int c = 0; c < 3; ++c) nv += V(dinv)[9 * node + 3 * l + c] * res[c];
        V(x)[3 * node + l] = (1 - w) * V(x)[3 * node + l] + w * nv;
      }
    }
  }

  void scale(DeviceVector &x, float a) override { HEnc e; encodeScale(e, x, a); }
  void scale(DeviceVector &x, const DeviceScalar &a) override { HEnc e; encodeScale(e, x, a); }
  void scaleVectorByVector(const DeviceVector &s, DeviceVector &y) override { HEnc e; encodeScaleVector(e, s, y); }
  void axpy(float a, const DeviceVector &x, DeviceVector &y) override { HEnc e; encodeAxpy(e, a, x, y); }
  void axpy(const DeviceScalar &a, const DeviceVector &x, DeviceVector &y) override { HEnc e; encodeAxpy(e, a, x, y); }
  void spmv(const DeviceCSRMatrix &A, const DeviceVector &x, DeviceVector &y) override { HEnc e; encodeSpmv(e, A, x, y); }
  void dot(const DeviceVector &x, const DeviceVector &y, DeviceScalar &r) override { HEnc e; encodeDot(e, x, y, r); }
  void scalarSet(float x, DeviceScalar &r) override { HEnc e; encodeScalarSet(e, x, r); }
  void scalarCopy(const DeviceScalar &a, DeviceScalar &o) override { HEnc e; encodeScalarCopy(e, a, o); }
  void scalarDivide(const DeviceScalar &a, const DeviceScalar &b, DeviceScalar &o) override {
    HEnc e;
    encodeScalarDivide(e, a, b, o);
  }
  void scalarMultiply(const DeviceScalar &a, const DeviceScalar &b, DeviceScalar &o) override {
    HEnc e;
    encodeScalarMultiply(e, a, b, o);
  }
  void scalarNegate(const DeviceScalar &a, DeviceScalar &o) override { HEnc e; encodeScalarNegate(e, a, o); }
  void scalarSqrt(const DeviceScalar &a, DeviceScalar &o) override { HEnc e; encodeScalarSqrt(e, a, o); }
};

}  // namespace hostbackend
