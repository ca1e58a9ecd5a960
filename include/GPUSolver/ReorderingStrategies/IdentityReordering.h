// gpuSolver::IdentityReordering (include/GPUSolver/ReorderingStrategies/
// IdentityReordering.h of the reference): oldToNew = newToOld = identity.
#pragma once
#include "ReorderingStrategy.h"

namespace gpuSolver {

class IdentityReordering : public ReorderingStrategy {
 public:
  void compute(std::size_t nRows, const int *, const int *, int *oldToNew, int *newToOld) const override {
    for (std::size_t i = 0; i < nRows; ++i) oldToNew[i] = newToOld[i] = static_cast<int>(i);
  }
};

}  // namespace gpuSolver
