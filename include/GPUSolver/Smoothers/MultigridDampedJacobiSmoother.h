// gpuSolver::MultigridDampedJacobiSmoother (include/GPUSolver/Smoothers/MultigridDampedJacobiSmoother.h of the reference),
// defined with MultigridSmoother.
#pragma once
#include "MultigridSmoother.h"
