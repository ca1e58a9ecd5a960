// gpuSolver::Backend (include/GPUSolver/Backend.h:15-159 of the reference):
// creates device objects and encodes the CG / smoother operations on them.
// Every encode* call appends to an encoder; the synchronous forms (spmv,
// dot, axpy, ...) encode on a temporary encoder and wait for it. The
// implementation on a B200 is gpuSolver::CudaBackend (= B200Backend,
// GPUSolver/cuda/CudaBackend.h).
//
// encodeBlockGaussSeidelColor3x3 reads its two range arguments as
// (colorStart, colorCount), the reading BlockGaussSeidelSmoother passes
// (src/Smoothers/BlockGaussSeidelSmoother.cc:149-166); the reference's CPU
// and CUDA backends read the second one as an end index, which only agrees
// for the first colour.
#pragma once
#include <cstddef>

namespace gpuSolver {

class BackendEncoder;
class DeviceVector;
class DeviceScalar;
class DeviceCSRMatrix;
class DeviceIndexVector;
class DeviceELLMatrix;
class HostCSRMatrix;
class HostELLMatrix;

class Backend {
 public:
  virtual ~Backend() = default;

  // the CUDA device the objects of this backend live on (no reference
  // counterpart: the reference's CudaBackend uses the current device)
  virtual int device() const { return 0; }

  virtual BackendEncoder *createEncoder() = 0;
  virtual void submit(BackendEncoder &encoder) = 0;
  virtual void submitAndWait(BackendEncoder &encoder) = 0;

  virtual DeviceVector *createVector(std::size_t size) = 0;
  virtual DeviceVector *createVector(std::size_t size, const float *values) = 0;
  virtual DeviceIndexVector *createIndexVector(std::size_t size) = 0;
  virtual DeviceIndexVector *createIndexVector(std::size_t size, const int *values) = 0;
  virtual DeviceScalar *createScalar() = 0;
  virtual DeviceScalar *createScalar(float value) = 0;
  virtual DeviceCSRMatrix *createCSRMatrix(const HostCSRMatrix &matrix) = 0;
  virtual DeviceELLMatrix *createELLMatrix(const HostELLMatrix &matrix) = 0;

  virtual void encodeScale(BackendEncoder &encoder, DeviceVector &x, float alpha) = 0;
  virtual void encodeScale(BackendEncoder &encoder, DeviceVector &x, const DeviceScalar &alpha) = 0;
  virtual void encodeCopy(BackendEncoder &encoder, const DeviceVector &x, DeviceVector &xCopy) = 0;
  virtual void encodeScaleVector(BackendEncoder &encoder, const DeviceVector &scaleVector,
                                 DeviceVector &output) = 0;
  virtual void encodeSetZero(BackendEncoder &encoder, DeviceVector &input) = 0;
  virtual void encodeAxpy(BackendEncoder &encoder, float alpha, const DeviceVector &x, DeviceVector &y) = 0;
  virtual void encodeAxpy(BackendEncoder &encoder, const DeviceScalar &alpha, const DeviceVector &x,
                          DeviceVector &y) = 0;
  virtual void encodeSpmv(BackendEncoder &encoder, const DeviceCSRMatrix &A, const DeviceVector &x,
                          DeviceVector &y) = 0;
  virtual void encodeGaussSeidelColor(BackendEncoder &encoder, const DeviceCSRMatrix &matrix,
                                      const DeviceIndexVector &colorVertices, std::size_t colorStart,
                                      std::size_t colorCount, const DeviceVector &rhs, DeviceVector &solution,
                                      float omega) = 0;
  virtual void encodeDot(BackendEncoder &encoder, const DeviceVector &x, const DeviceVector &y,
                         DeviceScalar &result) = 0;
  virtual void encodeScalarDivide(BackendEncoder &encoder, const DeviceScalar &numerator,
                                  const DeviceScalar &denominator, DeviceScalar &result) = 0;
  virtual void encodeScalarMultiply(BackendEncoder &encoder, const DeviceScalar &factor1,
                                    const DeviceScalar &factor2, DeviceScalar &result) = 0;
  virtual void encodeScalarSet(BackendEncoder &encoder, float value, DeviceScalar &output) = 0;
  virtual void encodeScalarCopy(BackendEncoder &encoder, const DeviceScalar &input, DeviceScalar &output) = 0;
  virtual void encodeScalarNegate(BackendEncoder &encoder, const DeviceScalar &input, DeviceScalar &output) = 0;
  virtual void encodeScalarSqrt(BackendEncoder &encoder, const DeviceScalar &input, DeviceScalar &output) = 0;
  virtual void encodeApplyBlockInverses3x3(BackendEncoder &encoder, const DeviceVector &inverseDiagBlocks,
                                           const DeviceVector &residual, DeviceVector &correction) = 0;
  virtual void encodeBlockGaussSeidelColor3x3(BackendEncoder &encoder, const DeviceCSRMatrix &matrix,
                                              const DeviceIndexVector &colorBlocks,
                                              const DeviceVector &diagonalInverses, std::size_t begin,
                                              std::size_t end, const DeviceVector &rhs, DeviceVector &solution,
                                              float omega) = 0;

  virtual void scale(DeviceVector &x, float alpha) = 0;
  virtual void scale(DeviceVector &x, const DeviceScalar &alpha) = 0;
  virtual void scaleVectorByVector(const DeviceVector &scaleVector, DeviceVector &output) = 0;
  virtual void axpy(float alpha, const DeviceVector &x, DeviceVector &y) = 0;
  virtual void axpy(const DeviceScalar &alpha, const DeviceVector &x, DeviceVector &y) = 0;
  virtual void spmv(const DeviceCSRMatrix &A, const DeviceVector &x, DeviceVector &y) = 0;
  virtual void dot(const DeviceVector &x, const DeviceVector &y, DeviceScalar &result) = 0;
  virtual void scalarSet(float value, DeviceScalar &result) = 0;
  virtual void scalarCopy(const DeviceScalar &input, DeviceScalar &output) = 0;
  virtual void scalarDivide(const DeviceScalar &numerator, const DeviceScalar &denominator,
                            DeviceScalar &result) = 0;
  virtual void scalarMultiply(const DeviceScalar &factor1, const DeviceScalar &factor2, DeviceScalar &result) = 0;
  virtual void scalarNegate(const DeviceScalar &input, DeviceScalar &output) = 0;
  virtual void scalarSqrt(const DeviceScalar &input, DeviceScalar &output) = 0;
};

}  // namespace gpuSolver
