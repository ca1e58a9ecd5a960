// gpuSolver::ReorderingStrategy (include/GPUSolver/ReorderingStrategies/
// ReorderingStrategy.h of the reference): computes a symmetric reordering of
// a CSR graph. The arguments are (oldToNew, newToOld), the order every
// implementation and caller of the reference uses (its base declaration
// names them the other way round).
#pragma once
#include "../detail/b200.h"

namespace gpuSolver {

class ReorderingStrategy {
 public:
  virtual ~ReorderingStrategy() = default;
  virtual void compute(std::size_t nRows, const int *rowPtr, const int *colPtr, int *oldToNew,
                       int *newToOld) const = 0;
};

}  // namespace gpuSolver
