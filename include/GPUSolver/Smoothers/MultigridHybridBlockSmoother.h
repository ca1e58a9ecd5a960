// gpuSolver::MultigridHybridBlockSmoother (include/GPUSolver/Smoothers/MultigridHybridBlockSmoother.h of the reference),
// defined with MultigridSmoother.
#pragma once
#include "MultigridSmoother.h"
