// gpuSolver::RCMReordering (src/ReorderingStrategies/RCMReordering.cc:11-110 of
// the reference): reverse Cuthill-McKee, bit-identical orderings.
#pragma once
#include "../detail/b200.h"

namespace gpuSolver {

class ReorderingStrategy {
 public:
  virtual ~ReorderingStrategy() = default;
  virtual void compute(std::size_t nRows, const int *rowPtr, const int *colPtr, int *oldToNew,
                       int *newToOld) const = 0;
};

class RCMReordering : public ReorderingStrategy {
 public:
  void compute(std::size_t nRows, const int *rowPtr, const int *colPtr, int *oldToNew,
               int *newToOld) const override {
    detail::check(gs_rcm(static_cast<int>(nRows), rowPtr, colPtr, oldToNew, newToOld));
  }
};

class IdentityReordering : public ReorderingStrategy {
 public:
  void compute(std::size_t nRows, const int *, const int *, int *oldToNew, int *newToOld) const override {
    for (std::size_t i = 0; i < nRows; ++i) oldToNew[i] = newToOld[i] = static_cast<int>(i);
  }
};

}  // namespace gpuSolver
