// gpuSolver::GraphColoring (include/GPUSolver/GraphColoring.h, src/GraphColoring.cc:9-72
// of the reference): greedy first-fit colouring in natural order.
#pragma once
#include <vector>

#include "detail/b200.h"

namespace gpuSolver {

class GraphColoring {
 public:
  void compute(std::size_t n, const int *rowPtr, const int *colPtr) {
    colors_.assign(n, 0);
    vertices_.assign(n, 0);
    offsets_.assign(n + 2, 0);
    int nc = 0;
    detail::check(gs_greedy_coloring(static_cast<int>(n), rowPtr, colPtr, colors_.data(),
                                     vertices_.data(), offsets_.data(), &nc));
    offsets_.resize(nc + 1);
    n_colors_ = nc;
    initialized_ = true;
  }
  std::size_t numberOfColors() const { return static_cast<std::size_t>(n_colors_); }
  const std::vector<int> &colors() const { return get(colors_); }
  const std::vector<int> &colorVertices() const { return get(vertices_); }
  const std::vector<int> &colorOffsets() const { return get(offsets_); }

 private:
  const std::vector<int> &get(const std::vector<int> &v) const {
    if (!initialized_) throw std::runtime_error(" the coloring was not initialized");
    return v;
  }
  std::vector<int> colors_, vertices_, offsets_;
  int n_colors_ = 0;
  bool initialized_ = false;
};

}  // namespace gpuSolver
