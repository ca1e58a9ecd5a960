// gpuSolver::Permutation (include/GPUSolver/Permutation.h of the reference).
#pragma once
#include "detail/b200.h"
