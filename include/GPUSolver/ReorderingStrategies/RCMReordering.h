// gpuSolver::RCMReordering (src/ReorderingStrategies/RCMReordering.cc:11-110 of
// the reference): reverse Cuthill-McKee, bit-identical orderings.
#pragma once
#include "IdentityReordering.h"
#include "ReorderingStrategy.h"

namespace gpuSolver {

class RCMReordering : public ReorderingStrategy {
 public:
  void compute(std::size_t nRows, const int *rowPtr, const int *colPtr, int *oldToNew,
               int *newToOld) const override {
    detail::check(gs_rcm(static_cast<int>(nRows), rowPtr, colPtr, oldToNew, newToOld));
  }
};

}  // namespace gpuSolver
