/**
 * @file fft_backend_b200.hpp
 * @brief B200Backend<T>: a ParaFaFT FFT backend running hand-written sm_100a
 *        kernels through the b200fft C ABI (b200fft.h).
 *
 * Satisfies the backend concept documented in ParaFaFT's
 * backend/fft_backend.hpp:45-196 and is a drop-in for the `Backend` template
 * parameter of ParaFaFT_C2C<D, Backend> (parafaft_c2c.hpp:69) and
 * ParaFaFT_R2C<D, Backend> (parafaft_r2c.hpp:98):
 *
 *   parafaft::ParaFaFT_R2C<3, parafaft::B200Backend<float>> fft(shape);
 *   fft.forward_in_place(device_buffer);   // same API, layout and results
 *
 * Method-by-method it mirrors CuFFTBackend (backend/cufft/fft_backend_cufft.hpp):
 * C2C stage plans and execution (:292-337), in-place padded R2C/C2R
 * (:360-469), asynchronous memcpy/memcpy2d on the backend stream and a
 * blocking sync (:483-519), device buffers with resize semantics (:58-121).
 * Errors throw std::runtime_error, as check_cuda/check_cufft do (:46-51,
 * :719-724).
 *
 * Differences a caller can observe:
 *  - Work the handle holds back for fusion (see b200fft.h) is issued at the
 *    next backend call that does not extend it, or at sync(). ParaFaFT calls
 *    sync() before every forward/backward returns (parafaft_r2c.hpp:429,541;
 *    parafaft_c2c.hpp:601,693). Setting B200FFT_NO_DEFER=1 in the
 *    environment (or B200FFT_FLAG_NO_DEFER through set_flags() before
 *    planning) issues every call immediately.
 *  - Plan arguments are 64-bit end to end (no int narrowing, unlike
 *    cufftPlanMany, fft_backend_cufft.hpp:673-689).
 *  - The backend is single-rank: use_p2p is false, so constructing it on a
 *    communicator with more than one rank throws (ParaFaFT would otherwise
 *    index its P2P table, sized only when use_p2p is true,
 *    parafaft_c2c.hpp:585,907-908).
 */
#ifndef PARAFAFT_BACKEND_B200_HPP
#define PARAFAFT_BACKEND_B200_HPP

#include <complex>
#include <cstddef>
#include <mpi.h>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "b200fft.h"

namespace parafaft {

#ifndef PARAFAFT_BACKEND_HPP
// Forward declarations of the concept's enums when this header is used
// without ParaFaFT's backend/fft_backend.hpp (same values, :25-43).
enum class FFTDirection { Forward, Backward };
enum class FFTPlanFlag { Estimate, Measure, Patient };
#endif

namespace b200_detail {
/// Handle of the B200Backend most recently constructed on this thread. The
/// orchestrators keep their backend private; instrumentation (launch counts,
/// fusion statistics) reads the handle from here right after construction.
inline b200fft_handle &last_opened() {
  static thread_local b200fft_handle h = nullptr;
  return h;
}
inline void check(int rc, const char *what) {
  if (rc != B200FFT_SUCCESS)
    throw std::runtime_error(std::string("B200 backend error in ") + what + ": " +
                             b200fft_last_error());
}
} // namespace b200_detail

/**
 * @brief Owning device vector (the Buffer/ComplexBuffer of B200Backend).
 *
 * Same semantics as cuvector<T> (fft_backend_cufft.hpp:58-121): resize()
 * discards the old contents; data() is a device pointer.
 */
template <typename T> class b200vector {
public:
  b200vector() = default;
  explicit b200vector(std::size_t n) { resize(n); }
  ~b200vector() { b200fft_free(data_); }
  b200vector(const b200vector &) = delete;
  b200vector &operator=(const b200vector &) = delete;
  b200vector(b200vector &&o) noexcept : data_(o.data_), size_(o.size_) {
    o.data_ = nullptr;
    o.size_ = 0;
  }
  b200vector &operator=(b200vector &&o) noexcept {
    if (this != &o) {
      b200fft_free(data_);
      data_ = o.data_;
      size_ = o.size_;
      o.data_ = nullptr;
      o.size_ = 0;
    }
    return *this;
  }
  void resize(std::size_t n) {
    if (n == size_)
      return;
    void *p = nullptr;
    b200_detail::check(b200fft_alloc(n * sizeof(T), &p), "b200vector::resize");
    b200fft_free(data_);
    data_ = static_cast<T *>(p);
    size_ = n;
  }
  T *data() { return data_; }
  const T *data() const { return data_; }
  std::size_t size() const { return size_; }

private:
  T *data_ = nullptr;
  std::size_t size_ = 0;
};

/**
 * @brief ParaFaFT backend on the B200 transform engine.
 * @tparam FloatTypeT float or double.
 */
template <typename FloatTypeT = double> class B200Backend {
  static_assert(std::is_same<FloatTypeT, float>::value ||
                    std::is_same<FloatTypeT, double>::value,
                "B200Backend supports float and double");

public:
  using FloatType = FloatTypeT;
  using Complex = std::complex<FloatType>;
  using Buffer = b200vector<FloatType>;
  using ComplexBuffer = b200vector<Complex>;

  static constexpr bool use_alltoallw = false;
  static constexpr bool handles_distributed = false;
  static constexpr bool use_p2p = false;

  explicit B200Backend(int num_stages, FFTPlanFlag plan_flag = FFTPlanFlag::Estimate)
      : num_stages_(num_stages), plan_flag_(plan_flag) {
    open();
  }

  explicit B200Backend(int num_stages, MPI_Comm comm,
                       FFTPlanFlag plan_flag = FFTPlanFlag::Estimate)
      : num_stages_(num_stages), plan_flag_(plan_flag) {
    int size = 1;
    MPI_Comm_size(comm, &size);
    if (size != 1)
      throw std::runtime_error(
          "B200Backend runs one rank per GPU without exchange: communicator has " +
          std::to_string(size) + " ranks");
    open();
  }

  ~B200Backend() { b200fft_destroy(h_); }

  B200Backend(const B200Backend &) = delete;
  B200Backend &operator=(const B200Backend &) = delete;
  B200Backend(B200Backend &&o) noexcept
      : num_stages_(o.num_stages_), plan_flag_(o.plan_flag_), flags_(o.flags_),
        h_(o.h_) {
    o.h_ = nullptr;
  }

  /// Handle creation flags (B200FFT_FLAG_*); recreates the handle, so call
  /// it before any plan is made.
  void set_flags(unsigned flags) {
    b200fft_destroy(h_);
    h_ = nullptr;
    flags_ = flags;
    open();
  }

  // ---- C2C (fft_backend_cufft.hpp:292-337) --------------------------------
  // With FFTPlanFlag::Measure/Patient the planning pointer (ParaFaFT's
  // scratch buffer) is where kernel candidates are timed; its contents are
  // overwritten, as with FFTW_MEASURE.
  void create_stage_plan(int stage, int length, std::size_t batch, Complex *data,
                         std::ptrdiff_t stride, std::ptrdiff_t dist) {
    planning_buffer(data);
    b200_detail::check(b200fft_plan_c2c(h_, stage, length, batch, stride, dist),
                       "create_stage_plan");
  }

  void execute_stage(int stage, FFTDirection direction, Complex *data) {
    b200_detail::check(
        b200fft_exec_c2c(h_, stage,
                         direction == FFTDirection::Forward ? B200FFT_FORWARD
                                                            : B200FFT_BACKWARD,
                         data),
        "execute_stage");
  }

  // ---- in-place R2C / C2R (fft_backend_cufft.hpp:360-469) -----------------
  void create_r2c_inplace_plan(int length, std::size_t batch, FloatType *padded_real,
                               std::ptrdiff_t stride, std::ptrdiff_t dist) {
    planning_buffer(padded_real);
    b200_detail::check(b200fft_plan_r2c(h_, length, batch, stride, dist),
                       "create_r2c_inplace_plan");
  }
  void execute_r2c_inplace(FloatType *padded_real) {
    b200_detail::check(b200fft_exec_r2c(h_, padded_real), "execute_r2c_inplace");
  }
  void create_c2r_inplace_plan(int length, std::size_t batch, FloatType *padded_real,
                               std::ptrdiff_t stride, std::ptrdiff_t dist) {
    planning_buffer(padded_real);
    b200_detail::check(b200fft_plan_c2r(h_, length, batch, stride, dist),
                       "create_c2r_inplace_plan");
  }
  void execute_c2r_inplace(FloatType *padded_real) {
    b200_detail::check(b200fft_exec_c2r(h_, padded_real), "execute_c2r_inplace");
  }

  // ---- copies and ordering (fft_backend_cufft.hpp:483-519) ----------------
  void memcpy(void *dest, const void *src, std::size_t bytes) const {
    b200_detail::check(b200fft_memcpy(h_, dest, src, bytes), "memcpy");
  }
  void memcpy2d(void *dst, std::size_t dpitch, const void *src, std::size_t spitch,
                std::size_t width, std::size_t height) const {
    b200_detail::check(b200fft_memcpy2d(h_, dst, dpitch, src, spitch, width, height),
                       "memcpy2d");
  }
  void sync() const { b200_detail::check(b200fft_sync(h_), "sync"); }
  /// No host NUMA placement for device memory (as CuFFTBackend).
  void first_touch(void * /*data*/, std::size_t /*bytes*/) const {}

  // ---- extras ----------------------------------------------------------------
  b200fft_handle handle() const { return h_; }
  b200fft_stats stats() const {
    b200fft_stats s{};
    b200_detail::check(b200fft_get_stats(h_, &s), "stats");
    return s;
  }

private:
  void planning_buffer(void *p) {
    if (plan_flag_ != FFTPlanFlag::Estimate)
      b200_detail::check(b200fft_set_work_buffer(h_, p, 0), "planning buffer");
  }

  void open() {
    const int prec = std::is_same<FloatType, double>::value ? B200FFT_F64 : B200FFT_F32;
    const int pf = plan_flag_ == FFTPlanFlag::Estimate
                       ? B200FFT_PLAN_ESTIMATE
                       : (plan_flag_ == FFTPlanFlag::Measure ? B200FFT_PLAN_MEASURE
                                                             : B200FFT_PLAN_PATIENT);
    b200_detail::check(b200fft_create(prec, num_stages_, pf, flags_, &h_), "construct");
    b200_detail::last_opened() = h_;
  }

  int num_stages_;
  FFTPlanFlag plan_flag_;
  unsigned flags_ = 0;
  b200fft_handle h_ = nullptr;
};

} // namespace parafaft

#endif // PARAFAFT_BACKEND_B200_HPP
