// gpuSolver::SymmetricGaussSeidelSmoother
// (src/Smoothers/SymmetricGaussSeidelSmoother.cc:12-128 of the reference):
// the greedy colouring of the active host matrix; one step is every colour
// forward, then every colour backward, each colour one encodeGaussSeidelColor
// with weight omega in (0, 2).
#pragma once
#include <cmath>
#include <memory>
#include <vector>

#include "../DeviceIndexVector.h"
#include "../GraphColoring.h"
#include "../Smoother.h"

namespace gpuSolver {

class SymmetricGaussSeidelSmoother : public Smoother {
 public:
  explicit SymmetricGaussSeidelSmoother(float omega = 1.0f) : omega_(omega) {
    if (!std::isfinite(omega_) || omega_ <= 0.0f || omega_ >= 2.0f)
      throw std::runtime_error("SymmetricGaussSeidelSmoother: invalid omega.");
  }
  SymmetricGaussSeidelSmoother(const SymmetricGaussSeidelSmoother &) = delete;
  SymmetricGaussSeidelSmoother &operator=(const SymmetricGaussSeidelSmoother &) = delete;

  void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) override {
    if (colorVertices_) throw std::runtime_error("SymmetricGaussSeidelSmoother: already initialized.");
    GraphColoring coloring;
    coloring.compute(hostMatrix.rows(), hostMatrix.activeRowPtr(), hostMatrix.activeColPtr());
    colorOffsets_ = coloring.colorOffsets();
    colorVertices_.reset(backend.createIndexVector(coloring.colorVertices().size(), coloring.colorVertices().data()));
    matrix_ = &deviceMatrix;
  }
  void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
              std::size_t iterations) override {
    if (matrix_ == nullptr || !colorVertices_)
      throw std::runtime_error("SymmetricGaussSeidelSmoother: not initialized.");
    if (iterations == 0) throw std::runtime_error("Preconditioner requires at least one smoothing step.");
    const std::size_t colors = colorOffsets_.size() - 1;
    auto pass = [&](std::size_t c) {
      const std::size_t begin = static_cast<std::size_t>(colorOffsets_[c]);
      const std::size_t count = static_cast<std::size_t>(colorOffsets_[c + 1]) - begin;
      backend.encodeGaussSeidelColor(encoder, *matrix_, *colorVertices_, begin, count, rhs, solution, omega_);
    };
    for (std::size_t it = 0; it < iterations; ++it) {
      for (std::size_t c = 0; c < colors; ++c) pass(c);
      for (std::size_t c = colors; c > 0; --c) pass(c - 1);
    }
  }
  const DeviceIndexVector &colorVertices() const { return *colorVertices_; }
  const std::vector<int> &colorOffsets() const { return colorOffsets_; }

 private:
  const DeviceCSRMatrix *matrix_ = nullptr;
  std::unique_ptr<DeviceIndexVector> colorVertices_;
  std::vector<int> colorOffsets_;
  float omega_;
};

}  // namespace gpuSolver
