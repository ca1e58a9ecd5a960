// gpuSolver::Backend / CudaBackend: the device the solvers run on.
#pragma once
#include "detail/b200.h"
