// gpuSolver::MultigridGaussSeidelSmoother (include/GPUSolver/Smoothers/MultigridGaussSeidelSmoother.h of the reference),
// defined with MultigridSmoother.
#pragma once
#include "MultigridSmoother.h"
