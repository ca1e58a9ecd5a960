// gpuSolver::Smoother (include/GPUSolver/Smoother.h of the reference): a
// relaxation that, once initialised with a matrix, applies `iterations`
// steps to `solution` for the right-hand side `rhs`, queued on an encoder.
// The single-level smoothers and the MultigridSmoother family
// (GPUSolver/Smoothers/) are built on the Backend operations; a full solve
// on a B200 goes through CGSolver and the Multigrid*Preconditioner classes,
// whose V-cycle runs fused on the device.
#pragma once
#include <cstddef>

#include "Backend.h"
#include "BackendEncoder.h"
#include "DeviceSparseMatrix.h"
#include "DeviceVector.h"
#include "HostSparseMatrix.h"

namespace gpuSolver {

class Smoother {
 public:
  virtual ~Smoother() = default;
  virtual void initialize(Backend &backend, const HostCSRMatrix &hostMatrix, const DeviceCSRMatrix &deviceMatrix) = 0;
  virtual void smooth(Backend &backend, BackendEncoder &encoder, const DeviceVector &rhs, DeviceVector &solution,
                      std::size_t iterations) = 0;
};

}  // namespace gpuSolver
