// gpuSolver::DampedJacobiSmoother (src/Smoothers/DampedJacobiSmoother.cc:5-89
// of the reference): x += omega D^-1 (b - A x) per step, D^-1 the FP32
// reciprocals of the first diagonal entry of each row (an entry below 1e-12
// in magnitude, or none, is an error).
#pragma once
#include <cmath>
#include <memory>
#include <vector>

#include "../Smoother.h"

namespace gpuSolver {

class DampedJacobiSmoother : public Smoother {
 public:
  explicit DampedJacobiSmoother(float omega = 0.7f) : omega_(omega) {}
  DampedJacobiSmoother(const DampedJacobiSmoother &) = delete;
  DampedJacobiSmoother &operator=(const DampedJacobiSmoother &) = delete;

  void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) override {
    if (inverseDiagonal_) throw std::runtime_error("DampedJacobiPreconditioner::initialize: already initialized.");
    const std::size_t n = hostMatrix.rows();
    const int *rp = hostMatrix.activeRowPtr();
    const int *ci = hostMatrix.activeColPtr();
    const float *v = hostMatrix.activeValPtr();
    std::vector<float> inv(n);
    for (std::size_t r = 0; r < n; ++r) {
      int k = rp[r];
      while (k < rp[r + 1] && ci[k] != static_cast<int>(r)) ++k;
      if (k == rp[r + 1]) throw std::runtime_error("DampedJacobiPreconditioner::initialize: missing diagonal entry.");
      if (std::fabs(v[k]) < 1e-12f)
        throw std::runtime_error("DampedJacobiPreconditioner::initialize: zero diagonal entry.");
      inv[r] = 1.0f / v[k];
    }
    inverseDiagonal_.reset(backend.createVector(n, inv.data()));
    Az_.reset(backend.createVector(n));
    correction_.reset(backend.createVector(n));
    matrix_ = &deviceMatrix;
  }
  void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
              std::size_t iterations) override {
    if (matrix_ == nullptr) throw std::runtime_error("DampedJacobiSmoother: not initialized.");
    for (std::size_t it = 0; it < iterations; ++it) {
      backend.encodeSpmv(encoder, *matrix_, solution, *Az_);
      backend.encodeCopy(encoder, rhs, *correction_);
      backend.encodeAxpy(encoder, -1.0f, *Az_, *correction_);
      backend.encodeScaleVector(encoder, *inverseDiagonal_, *correction_);
      backend.encodeAxpy(encoder, omega_, *correction_, solution);
    }
  }

 private:
  const DeviceCSRMatrix *matrix_ = nullptr;
  std::unique_ptr<DeviceVector> inverseDiagonal_, Az_, correction_;
  float omega_;
};

}  // namespace gpuSolver
