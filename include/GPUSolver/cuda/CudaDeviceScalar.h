// gpuSolver::CudaDeviceScalar (include/GPUSolver/cuda/CudaDeviceScalar.h of the reference): defined in
// CudaBackend.h as an alias of its B200 implementation.
#pragma once
#include "CudaBackend.h"
