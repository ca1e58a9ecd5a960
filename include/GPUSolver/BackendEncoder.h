// gpuSolver::BackendEncoder (include/GPUSolver/BackendEncoder.h of the
// reference): an ordered queue of device work; Backend::encode* calls append
// to it and Backend::submit / submitAndWait wait for it.
#pragma once

namespace gpuSolver {

class BackendEncoder {
 public:
  virtual ~BackendEncoder() = default;
  BackendEncoder(const BackendEncoder &) = delete;
  BackendEncoder &operator=(const BackendEncoder &) = delete;

 protected:
  BackendEncoder() = default;
};

}  // namespace gpuSolver
