// gpuSolver::CudaBackend on a B200 (src/cuda/CudaBackend.cc, src/cuda/CudaDevice*.cc
// and src/cuda/CudaEncoder.cc of the reference), header-only over the
// gpusolver_b200 C ABI: FP32 device objects, one blocking CUDA stream per
// encoder, the kernel-level entry points (gs_spmv, gs_gauss_seidel_color, ...)
// for the operations. Shapes and colour ranges are checked on the host
// before anything is queued; every failure throws std::runtime_error.
//
// Differences kept on purpose: the synchronous forms (spmv, dot, ...) wait
// for their temporary encoder before returning (the reference's destroy it
// with the work possibly still queued); scalarSet sets the scalar and
// returns (the reference's throws "not implemented yet" after doing the
// work); createELLMatrix uploads the ELL arrays (the reference's CUDA
// backend throws "not implemented yet"; no CUDA operation reads an ELL
// matrix in either). Device CSR matrices are created on the calling
// thread's current device, the other objects on the backend's device.
#pragma once
#include <memory>
#include <string>

#include "../Backend.h"
#include "../BackendEncoder.h"
#include "../DeviceELLMatrix.h"
#include "../DeviceIndexVector.h"
#include "../DeviceScalar.h"
#include "../DeviceSparseMatrix.h"
#include "../DeviceVector.h"
#include "../HostELLMatrix.h"
#include "../HostSparseMatrix.h"
#include "../detail/b200.h"

namespace gpuSolver {
namespace detail {

// One device allocation (gs_device_malloc / gs_device_free).
class DeviceMemory {
 public:
  DeviceMemory() = default;
  DeviceMemory(int device, std::size_t bytes) { check(gs_device_malloc(device, bytes, &p_)); }
  ~DeviceMemory() { reset(); }
  DeviceMemory(DeviceMemory &&o) noexcept : p_(o.p_) { o.p_ = nullptr; }
  DeviceMemory &operator=(DeviceMemory &&o) noexcept {
    if (this != &o) {
      reset();
      p_ = o.p_;
      o.p_ = nullptr;
    }
    return *this;
  }
  DeviceMemory(const DeviceMemory &) = delete;
  DeviceMemory &operator=(const DeviceMemory &) = delete;
  void *get() const { return p_; }

 private:
  void reset() {
    if (p_) gs_device_free(p_);
    p_ = nullptr;
  }
  void *p_ = nullptr;
};

inline void to_device(void *dst, const void *src, std::size_t bytes) {
  check(gs_memcpy(dst, src, bytes, GS_COPY_H2D, nullptr));
}
inline void to_host(void *dst, const void *src, std::size_t bytes) {
  check(gs_memcpy(dst, src, bytes, GS_COPY_D2H, nullptr));
}

// A typed device array with the reference's updateValues / download rules.
template <typename T>
class DeviceArray {
 public:
  DeviceArray(int device, std::size_t n) : device_(device), n_(n), mem_(device, n * sizeof(T)) {
    check(gs_memset(mem_.get(), 0, n * sizeof(T), nullptr));
  }
  std::size_t size() const { return n_; }
  T *data() const { return static_cast<T *>(mem_.get()); }
  // same size: new values in place; another size: a new allocation
  void update(const T *values, std::size_t n) {
    if (n > 0 && values == nullptr) throw std::runtime_error("updateValues: values must not be null.");
    if (n != n_) {
      DeviceMemory m(device_, n * sizeof(T));
      to_device(m.get(), values, n * sizeof(T));
      mem_ = std::move(m);
      n_ = n;
      return;
    }
    to_device(mem_.get(), values, n * sizeof(T));
  }
  T *download() const {
    host_.resize(n_);
    to_host(host_.data(), mem_.get(), n_ * sizeof(T));
    return host_.data();
  }

 private:
  int device_;
  std::size_t n_;
  DeviceMemory mem_;
  mutable std::vector<T> host_;
};

}  // namespace detail

class B200Encoder : public BackendEncoder {
 public:
  explicit B200Encoder(int device) { detail::check(gs_stream_create(device, &stream_)); }
  ~B200Encoder() override {
    if (stream_) gs_stream_destroy(stream_);
  }
  void *stream() const { return stream_; }

 private:
  void *stream_ = nullptr;
};

class B200DeviceVector : public DeviceVector {
 public:
  B200DeviceVector(int device, std::size_t size) : a_(device, size) {}
  std::size_t size() const override { return a_.size(); }
  void updateValues(const float *values, std::size_t sizeOfValues) override { a_.update(values, sizeOfValues); }
  float *download() const override { return a_.download(); }
  float *data() const { return a_.data(); }

 private:
  detail::DeviceArray<float> a_;
};

class B200DeviceIndexVector : public DeviceIndexVector {
 public:
  B200DeviceIndexVector(int device, std::size_t size) : a_(device, size) {}
  std::size_t size() const override { return a_.size(); }
  void updateValues(const int *values, std::size_t sizeOfValues) override { a_.update(values, sizeOfValues); }
  int *download() const override { return a_.download(); }
  int *data() const { return a_.data(); }

 private:
  detail::DeviceArray<int> a_;
};

class B200DeviceScalar : public DeviceScalar {
 public:
  B200DeviceScalar(int device, float value) : a_(device, 1) { a_.update(&value, 1); }
  float download() const override { return *a_.download(); }
  float *data() const { return a_.data(); }

 private:
  detail::DeviceArray<float> a_;
};

class B200DeviceCSRMatrix : public DeviceCSRMatrix {
 public:
  explicit B200DeviceCSRMatrix(const HostCSRMatrix &m) : rows_(m.rows()), cols_(m.cols()), nnz_(m.nnz()) {
    detail::check(gs_device_csr_create(static_cast<int>(rows_), static_cast<int>(cols_), m.activeRowPtr(),
                                       m.activeColPtr(), m.activeValPtr(), GS_F32, &h_));
  }
  ~B200DeviceCSRMatrix() override {
    if (h_) gs_device_csr_destroy(h_);
  }
  std::size_t rows() const override { return rows_; }
  std::size_t cols() const override { return cols_; }
  std::size_t nnz() const override { return nnz_; }
  void updateValues(const float *values, std::size_t numberOfValues) override {
    detail::check(gs_device_csr_update_values(h_, values, static_cast<long long>(numberOfValues)));
  }
  const gs_device_csr *handle() const { return h_; }

 private:
  std::size_t rows_, cols_, nnz_;
  gs_device_csr *h_ = nullptr;
};

class B200DeviceELLMatrix : public DeviceELLMatrix {
 public:
  B200DeviceELLMatrix(int device, const HostELLMatrix &m)
      : rows_(m.rows()), cols_(m.cols()), width_(m.ellWidth()), ovf_(m.overflowNnz()),
        col_(device, rows_ * width_), val_(device, rows_ * width_), orp_(device, rows_ + 1), oci_(device, ovf_),
        ov_(device, ovf_) {
    col_.update(m.ellColIdx(), rows_ * width_);
    val_.update(m.ellValues(), rows_ * width_);
    orp_.update(m.overflowRowPtr(), rows_ + 1);
    if (ovf_ > 0) {
      oci_.update(m.overflowColIdx(), ovf_);
      ov_.update(m.overflowValues(), ovf_);
    }
  }
  std::size_t rows() const override { return rows_; }
  std::size_t cols() const override { return cols_; }
  std::size_t ellWidth() const override { return width_; }
  std::size_t overflowNnz() const override { return ovf_; }
  const int *ellColIdx() const { return col_.data(); }
  const float *ellValues() const { return val_.data(); }
  const int *overflowRowPtr() const { return orp_.data(); }
  const int *overflowColIdx() const { return oci_.data(); }
  const float *overflowValues() const { return ov_.data(); }

 private:
  std::size_t rows_, cols_, width_, ovf_;
  detail::DeviceArray<int> col_;
  detail::DeviceArray<float> val_;
  detail::DeviceArray<int> orp_, oci_;
  detail::DeviceArray<float> ov_;
};

class B200Backend : public Backend {
 public:
  explicit B200Backend(int device = 0) : device_(device) {}
  int device() const override { return device_; }

  BackendEncoder *createEncoder() override { return new B200Encoder(device_); }
  void submit(BackendEncoder &encoder) override { detail::check(gs_stream_synchronize(stream(encoder))); }
  void submitAndWait(BackendEncoder &encoder) override { detail::check(gs_stream_synchronize(stream(encoder))); }

  DeviceVector *createVector(std::size_t size) override { return new B200DeviceVector(device_, size); }
  DeviceVector *createVector(std::size_t size, const float *values) override {
    std::unique_ptr<B200DeviceVector> v(new B200DeviceVector(device_, size));
    v->updateValues(values, size);
    return v.release();
  }
  DeviceIndexVector *createIndexVector(std::size_t size) override { return new B200DeviceIndexVector(device_, size); }
  DeviceIndexVector *createIndexVector(std::size_t size, const int *values) override {
    std::unique_ptr<B200DeviceIndexVector> v(new B200DeviceIndexVector(device_, size));
    v->updateValues(values, size);
    return v.release();
  }
  DeviceScalar *createScalar() override { return new B200DeviceScalar(device_, 0.0f); }
  DeviceScalar *createScalar(float value) override { return new B200DeviceScalar(device_, value); }
  DeviceCSRMatrix *createCSRMatrix(const HostCSRMatrix &matrix) override { return new B200DeviceCSRMatrix(matrix); }
  DeviceELLMatrix *createELLMatrix(const HostELLMatrix &matrix) override {
    return new B200DeviceELLMatrix(device_, matrix);
  }

  void encodeScale(BackendEncoder &e, DeviceVector &x, float alpha) override {
    vec(e, GS_VEC_SCALE, x.size(), nullptr, x, alpha, nullptr);
  }
  void encodeScale(BackendEncoder &e, DeviceVector &x, const DeviceScalar &alpha) override {
    vec(e, GS_VEC_SCALE, x.size(), nullptr, x, 0.0, &alpha);
  }
  void encodeCopy(BackendEncoder &e, const DeviceVector &x, DeviceVector &xCopy) override {
    same_size(x, xCopy, "encodeCopy");
    vec(e, GS_VEC_COPY, x.size(), &x, xCopy, 0.0, nullptr);
  }
  void encodeScaleVector(BackendEncoder &e, const DeviceVector &scaleVector, DeviceVector &output) override {
    same_size(scaleVector, output, "encodeScaleVector");
    vec(e, GS_VEC_SCALE_BY_VECTOR, output.size(), &scaleVector, output, 0.0, nullptr);
  }
  void encodeSetZero(BackendEncoder &e, DeviceVector &input) override {
    vec(e, GS_VEC_SET_ZERO, input.size(), nullptr, input, 0.0, nullptr);
  }
  void encodeAxpy(BackendEncoder &e, float alpha, const DeviceVector &x, DeviceVector &y) override {
    same_size(x, y, "encodeAxpy");
    vec(e, GS_VEC_AXPY, y.size(), &x, y, alpha, nullptr);
  }
  void encodeAxpy(BackendEncoder &e, const DeviceScalar &alpha, const DeviceVector &x, DeviceVector &y) override {
    same_size(x, y, "encodeAxpy");
    vec(e, GS_VEC_AXPY, y.size(), &x, y, 0.0, &alpha);
  }
  void encodeSpmv(BackendEncoder &e, const DeviceCSRMatrix &A, const DeviceVector &x, DeviceVector &y) override {
    if (x.size() != A.cols() || y.size() != A.rows()) throw std::runtime_error("encodeSpmv: dimension mismatch.");
    detail::check(gs_spmv(csr(A), vdata(x), vdata(y), stream(e)));
  }
  void encodeGaussSeidelColor(BackendEncoder &e, const DeviceCSRMatrix &matrix,
                              const DeviceIndexVector &colorVertices, std::size_t colorStart, std::size_t colorCount,
                              const DeviceVector &rhs, DeviceVector &solution, float omega) override {
    if (rhs.size() != matrix.rows() || solution.size() != matrix.rows())
      throw std::runtime_error("encodeGaussSeidelColor: dimension mismatch.");
    if (colorStart + colorCount > colorVertices.size())
      throw std::runtime_error("encodeGaussSeidelColor: invalid color range.");
    detail::check(gs_gauss_seidel_color(csr(matrix), idata(colorVertices), static_cast<long long>(colorStart),
                                        static_cast<long long>(colorCount), vdata(rhs), vdata(solution), omega,
                                        stream(e)));
  }
  void encodeDot(BackendEncoder &e, const DeviceVector &x, const DeviceVector &y, DeviceScalar &result) override {
    same_size(x, y, "encodeDot");
    detail::check(gs_dot(static_cast<long long>(x.size()), vdata(x), vdata(y), sdata(result), GS_F32, stream(e)));
  }
  void encodeScalarDivide(BackendEncoder &e, const DeviceScalar &numerator, const DeviceScalar &denominator,
                          DeviceScalar &result) override {
    sc(e, GS_SCALAR_DIVIDE, &numerator, &denominator, result, 0.0);
  }
  void encodeScalarMultiply(BackendEncoder &e, const DeviceScalar &factor1, const DeviceScalar &factor2,
                            DeviceScalar &result) override {
    sc(e, GS_SCALAR_MULTIPLY, &factor1, &factor2, result, 0.0);
  }
  void encodeScalarSet(BackendEncoder &e, float value, DeviceScalar &output) override {
    sc(e, GS_SCALAR_SET, nullptr, nullptr, output, value);
  }
  void encodeScalarCopy(BackendEncoder &e, const DeviceScalar &input, DeviceScalar &output) override {
    sc(e, GS_SCALAR_COPY, &input, nullptr, output, 0.0);
  }
  void encodeScalarNegate(BackendEncoder &e, const DeviceScalar &input, DeviceScalar &output) override {
    sc(e, GS_SCALAR_NEGATE, &input, nullptr, output, 0.0);
  }
  void encodeScalarSqrt(BackendEncoder &e, const DeviceScalar &input, DeviceScalar &output) override {
    sc(e, GS_SCALAR_SQRT, &input, nullptr, output, 0.0);
  }
  void encodeApplyBlockInverses3x3(BackendEncoder &e, const DeviceVector &inverseDiagBlocks,
                                   const DeviceVector &residual, DeviceVector &correction) override {
    same_size(residual, correction, "encodeApplyBlockInverses3x3");
    if (inverseDiagBlocks.size() != 3 * residual.size())
      throw std::runtime_error("encodeApplyBlockInverses3x3: expected 9 inverse entries per node.");
    detail::check(gs_apply_block_inverses3x3(static_cast<long long>(residual.size()), vdata(inverseDiagBlocks),
                                             vdata(residual), vdata(correction), GS_F32, stream(e)));
  }
  void encodeBlockGaussSeidelColor3x3(BackendEncoder &e, const DeviceCSRMatrix &matrix,
                                      const DeviceIndexVector &colorBlocks, const DeviceVector &diagonalInverses,
                                      std::size_t begin, std::size_t end, const DeviceVector &rhs,
                                      DeviceVector &solution, float omega) override {
    const std::size_t count = end;  // (colorStart, colorCount), see Backend.h
    if (rhs.size() != matrix.rows() || solution.size() != matrix.rows() ||
        diagonalInverses.size() != 3 * matrix.rows())
      throw std::runtime_error("encodeBlockGaussSeidelColor3x3: dimension mismatch.");
    if (begin + count > colorBlocks.size())
      throw std::runtime_error("encodeBlockGaussSeidelColor3x3: invalid color range.");
    detail::check(gs_block_gauss_seidel_color3x3(csr(matrix), idata(colorBlocks), static_cast<long long>(begin),
                                                 static_cast<long long>(count), vdata(diagonalInverses), vdata(rhs),
                                                 vdata(solution), omega, stream(e)));
  }

  void scale(DeviceVector &x, float alpha) override {
    once([&](BackendEncoder &e) { encodeScale(e, x, alpha); });
  }
  void scale(DeviceVector &x, const DeviceScalar &alpha) override {
    once([&](BackendEncoder &e) { encodeScale(e, x, alpha); });
  }
  void scaleVectorByVector(const DeviceVector &scaleVector, DeviceVector &output) override {
    once([&](BackendEncoder &e) { encodeScaleVector(e, scaleVector, output); });
  }
  void axpy(float alpha, const DeviceVector &x, DeviceVector &y) override {
    once([&](BackendEncoder &e) { encodeAxpy(e, alpha, x, y); });
  }
  void axpy(const DeviceScalar &alpha, const DeviceVector &x, DeviceVector &y) override {
    once([&](BackendEncoder &e) { encodeAxpy(e, alpha, x, y); });
  }
  void spmv(const DeviceCSRMatrix &A, const DeviceVector &x, DeviceVector &y) override {
    once([&](BackendEncoder &e) { encodeSpmv(e, A, x, y); });
  }
  void dot(const DeviceVector &x, const DeviceVector &y, DeviceScalar &result) override {
    once([&](BackendEncoder &e) { encodeDot(e, x, y, result); });
  }
  void scalarSet(float value, DeviceScalar &result) override {
    once([&](BackendEncoder &e) { encodeScalarSet(e, value, result); });
  }
  void scalarCopy(const DeviceScalar &input, DeviceScalar &output) override {
    once([&](BackendEncoder &e) { encodeScalarCopy(e, input, output); });
  }
  void scalarDivide(const DeviceScalar &numerator, const DeviceScalar &denominator, DeviceScalar &result) override {
    once([&](BackendEncoder &e) { encodeScalarDivide(e, numerator, denominator, result); });
  }
  void scalarMultiply(const DeviceScalar &factor1, const DeviceScalar &factor2, DeviceScalar &result) override {
    once([&](BackendEncoder &e) { encodeScalarMultiply(e, factor1, factor2, result); });
  }
  void scalarNegate(const DeviceScalar &input, DeviceScalar &output) override {
    once([&](BackendEncoder &e) { encodeScalarNegate(e, input, output); });
  }
  void scalarSqrt(const DeviceScalar &input, DeviceScalar &output) override {
    once([&](BackendEncoder &e) { encodeScalarSqrt(e, input, output); });
  }

 private:
  // Objects of another backend implementation cannot be used here.
  template <typename Impl, typename Base>
  static const Impl &as(const Base &b, const char *what) {
    const Impl *p = dynamic_cast<const Impl *>(&b);
    if (p == nullptr) throw std::runtime_error(std::string(what) + " was not created by a CudaBackend.");
    return *p;
  }
  static void *stream(BackendEncoder &e) { return as<B200Encoder>(e, "encoder").stream(); }
  static float *vdata(const DeviceVector &v) { return as<B200DeviceVector>(v, "vector").data(); }
  static int *idata(const DeviceIndexVector &v) { return as<B200DeviceIndexVector>(v, "index vector").data(); }
  static float *sdata(const DeviceScalar &s) { return as<B200DeviceScalar>(s, "scalar").data(); }
  static const gs_device_csr *csr(const DeviceCSRMatrix &m) { return as<B200DeviceCSRMatrix>(m, "matrix").handle(); }
  static void same_size(const DeviceVector &a, const DeviceVector &b, const char *what) {
    if (a.size() != b.size()) throw std::runtime_error(std::string(what) + ": vector sizes differ.");
  }
  void vec(BackendEncoder &e, int op, std::size_t n, const DeviceVector *x, DeviceVector &y, double alpha,
           const DeviceScalar *alphaDev) {
    detail::check(gs_vector_op(op, static_cast<long long>(n), x ? vdata(*x) : nullptr, vdata(y), alpha,
                               alphaDev ? sdata(*alphaDev) : nullptr, GS_F32, stream(e)));
  }
  void sc(BackendEncoder &e, int op, const DeviceScalar *a, const DeviceScalar *b, DeviceScalar &out, double value) {
    detail::check(gs_scalar_op(op, a ? sdata(*a) : nullptr, b ? sdata(*b) : nullptr, sdata(out), value, GS_F32,
                               stream(e)));
  }
  template <typename F>
  void once(F &&f) {
    std::unique_ptr<BackendEncoder> e(createEncoder());
    f(*e);
    submitAndWait(*e);
  }

  int device_;
};

// the reference's class names (src/cuda/*.cc), so that code naming them compiles unchanged
using CudaBackend = B200Backend;
using CudaEncoder = B200Encoder;
using CudaDeviceVector = B200DeviceVector;
using CudaDeviceIndexVector = B200DeviceIndexVector;
using CudaDeviceScalar = B200DeviceScalar;
using CudaDeviceCSRMatrix = B200DeviceCSRMatrix;

}  // namespace gpuSolver
