// gpuSolver::BlockGaussSeidelSmoother
// (src/Smoothers/BlockGaussSeidelSmoother.cc:8-210 of the reference): 3x3
// block symmetric Gauss-Seidel on the greedy colouring of the node graph
// (buildBlockGraph), with the inverted diagonal blocks; one step is every
// node colour forward, then backward. The colour ranges are passed as
// (colorStart, colorCount), the reading the reference's smoother intends.
#pragma once
#include <memory>
#include <vector>

#include "../BlockUtils.h"
#include "../DeviceIndexVector.h"
#include "../GraphColoring.h"
#include "../Smoother.h"

namespace gpuSolver {

class BlockGaussSeidelSmoother : public Smoother {
 public:
  explicit BlockGaussSeidelSmoother(float omega = 1.0f) : omega_(omega) {
    if (omega_ <= 0.0f || omega_ >= 2.0f) throw std::runtime_error("BlockGaussSeidelSmoother: omega must be in (0, 2).");
  }
  BlockGaussSeidelSmoother(const BlockGaussSeidelSmoother &) = delete;
  BlockGaussSeidelSmoother &operator=(const BlockGaussSeidelSmoother &) = delete;

  void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) override {
    if (matrix_ != nullptr) throw std::runtime_error("BlockGaussSeidelSmoother: already initialized.");
    if (hostMatrix.rows() % 3 != 0)
      throw std::runtime_error("BlockGaussSeidelSmoother: number of DOFs must be divisible by 3.");
    const std::vector<float> inverses = extractInverseDiagonalBlocks3x3(hostMatrix);
    inverseDiagonalBlocks_.reset(backend.createVector(inverses.size(), inverses.data()));
    const BlockGraph graph = buildBlockGraph(hostMatrix, 3);
    GraphColoring coloring;
    coloring.compute(graph.rowPtr.size() - 1, graph.rowPtr.data(), graph.colPtr.data());
    colorOffsets_ = coloring.colorOffsets();
    colorBlocks_.reset(backend.createIndexVector(coloring.colorVertices().size(), coloring.colorVertices().data()));
    matrix_ = &deviceMatrix;
  }
  void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
              std::size_t iterations) override {
    if (matrix_ == nullptr) throw std::runtime_error("BlockGaussSeidelSmoother: not initialized.");
    if (iterations == 0) throw std::runtime_error("Preconditioner requires at least one smoothing step.");
    const std::size_t colors = colorOffsets_.size() - 1;
    auto pass = [&](std::size_t c) {
      const std::size_t begin = static_cast<std::size_t>(colorOffsets_[c]);
      const std::size_t count = static_cast<std::size_t>(colorOffsets_[c + 1]) - begin;
      backend.encodeBlockGaussSeidelColor3x3(encoder, *matrix_, *colorBlocks_, *inverseDiagonalBlocks_, begin, count,
                                             rhs, solution, omega_);
    };
    for (std::size_t it = 0; it < iterations; ++it) {
      for (std::size_t c = 0; c < colors; ++c) pass(c);
      for (std::size_t c = colors; c > 0; --c) pass(c - 1);
    }
  }

 private:
  const DeviceCSRMatrix *matrix_ = nullptr;
  std::unique_ptr<DeviceVector> inverseDiagonalBlocks_;
  std::unique_ptr<DeviceIndexVector> colorBlocks_;
  std::vector<int> colorOffsets_;
  float omega_;
};

}  // namespace gpuSolver
