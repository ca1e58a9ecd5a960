// gpuSolver::DeviceIndexVector (include/GPUSolver/DeviceIndexVector.h of the
// reference): an int32 vector in device memory (colour-grouped vertex
// lists); download() semantics as for DeviceVector.
#pragma once
#include <cstddef>

namespace gpuSolver {

class DeviceIndexVector {
 public:
  virtual ~DeviceIndexVector() = default;
  DeviceIndexVector(const DeviceIndexVector &) = delete;
  DeviceIndexVector &operator=(const DeviceIndexVector &) = delete;
  virtual std::size_t size() const = 0;
  virtual void updateValues(const int *values, std::size_t sizeOfValues) = 0;
  virtual int *download() const = 0;

 protected:
  DeviceIndexVector() = default;
};

}  // namespace gpuSolver
