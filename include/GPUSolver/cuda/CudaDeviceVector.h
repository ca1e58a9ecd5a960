// gpuSolver::CudaDeviceVector (include/GPUSolver/cuda/CudaDeviceVector.h of the reference): defined in
// CudaBackend.h as an alias of its B200 implementation.
#pragma once
#include "CudaBackend.h"
