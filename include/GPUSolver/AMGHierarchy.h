// gpuSolver::AMGHierarchy (include/GPUSolver/AMGHierarchy.h of the reference).
#pragma once
#include "detail/b200.h"
