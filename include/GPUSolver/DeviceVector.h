// gpuSolver::DeviceVector (include/GPUSolver/DeviceVector.h of the
// reference): an FP32 vector in device memory. download() copies it into a
// host buffer owned by the vector and returns that buffer (valid until the
// next download or the vector's destruction); updateValues with a new size
// reallocates (src/cuda/CudaDeviceVector.cc:51-100).
#pragma once
#include <cstddef>

namespace gpuSolver {

class DeviceVector {
 public:
  virtual ~DeviceVector() = default;
  virtual std::size_t size() const = 0;
  virtual void updateValues(const float *values, std::size_t sizeOfValues) = 0;
  virtual float *download() const = 0;
  DeviceVector(const DeviceVector &) = delete;
  DeviceVector &operator=(const DeviceVector &) = delete;

 protected:
  DeviceVector() = default;
};

}  // namespace gpuSolver
