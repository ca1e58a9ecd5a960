// gpuSolver::BlockJacobiSmoother (src/Smoothers/BlockJacobiSmoother.cc:5-87
// of the reference): x += omega D^-1 (b - A x) per step with D the 3x3
// diagonal blocks (extractInverseDiagonalBlocks3x3).
#pragma once
#include <memory>
#include <vector>

#include "../BlockUtils.h"
#include "../Smoother.h"

namespace gpuSolver {

class BlockJacobiSmoother : public Smoother {
 public:
  explicit BlockJacobiSmoother(float omega) : omega_(omega) {}
  BlockJacobiSmoother(const BlockJacobiSmoother &) = delete;
  BlockJacobiSmoother &operator=(const BlockJacobiSmoother &) = delete;

  void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) override {
    const std::vector<float> inverses = extractInverseDiagonalBlocks3x3(hostMatrix);
    const std::size_t n = hostMatrix.rows();
    inverseDiagonalBlocks_.reset(backend.createVector(inverses.size(), inverses.data()));
    Az_.reset(backend.createVector(n));
    residual_.reset(backend.createVector(n));
    correction_.reset(backend.createVector(n));
    matrix_ = &deviceMatrix;
  }
  void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
              std::size_t iterations) override {
    if (matrix_ == nullptr) throw std::runtime_error("BlockJacobiSmoother: not initialized.");
    for (std::size_t it = 0; it < iterations; ++it) {
      backend.encodeSpmv(encoder, *matrix_, solution, *Az_);
      backend.encodeCopy(encoder, rhs, *residual_);
      backend.encodeAxpy(encoder, -1.0f, *Az_, *residual_);
      backend.encodeApplyBlockInverses3x3(encoder, *inverseDiagonalBlocks_, *residual_, *correction_);
      backend.encodeAxpy(encoder, omega_, *correction_, solution);
    }
  }

 private:
  const DeviceCSRMatrix *matrix_ = nullptr;
  std::unique_ptr<DeviceVector> inverseDiagonalBlocks_, Az_, residual_, correction_;
  float omega_;
};

}  // namespace gpuSolver
