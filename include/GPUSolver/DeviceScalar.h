// gpuSolver::DeviceScalar (include/GPUSolver/DeviceScalar.h of the
// reference): one FP32 value in device memory; download() waits for the
// copy, so work that writes it must have been submitted first.
#pragma once

namespace gpuSolver {

class DeviceScalar {
 public:
  virtual ~DeviceScalar() = default;
  DeviceScalar(const DeviceScalar &) = delete;
  DeviceScalar &operator=(const DeviceScalar &) = delete;
  virtual float download() const = 0;

 protected:
  DeviceScalar() = default;
};

}  // namespace gpuSolver
