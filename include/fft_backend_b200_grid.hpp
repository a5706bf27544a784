/**
 * @file fft_backend_b200_grid.hpp
 * @brief B200GridBackend<D, T>: a ParaFaFT backend that owns the whole grid
 *        (handles_distributed = true) on one GPU.
 *
 * The single-GPU counterpart of ParaFaFT's cuFFTMp backend
 * (backend/cufft/fft_backend_cufftmp.hpp:67-348), behind the optional
 * "distributed transform" part of the backend concept
 * (backend/fft_backend.hpp:153-190). With it, ParaFaFT_C2C / ParaFaFT_R2C
 * delegate the whole transform to the backend (parafaft_c2c.hpp:122-149,
 * :539-543, :632-636; parafaft_r2c.hpp:144-185, :360-364, :473-477):
 *
 *   parafaft::ParaFaFT_C2C<3, parafaft::B200GridBackend<3, float>> fft(shape);
 *   auto *grid = fft.get_buffer();    // write the input here (device memory)
 *   fft.forward(nullptr);             // transforms the backend's buffer
 *
 * What the backend does with it, B200-first:
 *  - every axis pass runs in place on the backend's own buffer: no scratch
 *    buffer and no exchange copies (the per-stage path needs two buffers);
 *  - each of the four transforms (C2C forward and backward, R2C forward, C2R
 *    backward) is planned once on its own b200fft handle, its passes are
 *    recorded once as a b200fft group (the middle-axis slice loops coalesce
 *    into one launch per axis) and captured in a CUDA graph; forward() and
 *    friends replay that graph and wait for it, so a transform costs one
 *    graph launch and one synchronisation instead of a host loop of
 *    per-stage and per-slice calls.
 *
 * Layouts (one rank: every start is 0, every local shape the global one):
 *  - C2C buffer (get_buffer): [N0]...[N_{D-1}] complex, row-major;
 *  - R2C buffer (get_real_buffer): [N0]...[N_{D-2}][2*(N_{D-1}/2+1)] reals,
 *    ParaFaFT's padded in-place layout (parafaft_r2c.hpp:804-847); after the
 *    forward transform it holds [N0]...[N_{D-2}][N_{D-1}/2+1] complex.
 * Each side is set up on first use: get_buffer()/forward()/backward()
 * allocate and plan the C2C grid, get_real_buffer()/forward_r2c()/
 * backward_c2r() the R2C one, so an object holds only the grid its
 * orchestrator transforms. As with cuFFTMp, get_distributed_info() describes
 * the C2C grid (required_size in complex elements).
 *
 * Results are those of B200Backend<T> through the per-stage path (the same
 * kernels on the same passes); transforms are unnormalised.
 *
 * One rank only: setup_distributed() throws on a communicator of more than
 * one rank.
 */
#ifndef PARAFAFT_BACKEND_B200_GRID_HPP
#define PARAFAFT_BACKEND_B200_GRID_HPP

#include <array>
#include <cstddef>
#include <mpi.h>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "fft_backend_b200.hpp"

namespace parafaft {

template <int D, typename FloatTypeT = double> class B200GridBackend {
  static_assert(D >= 2, "B200GridBackend needs at least two axes");
  static_assert(std::is_same<FloatTypeT, float>::value ||
                    std::is_same<FloatTypeT, double>::value,
                "B200GridBackend supports float and double");

public:
  using FloatType = FloatTypeT;
  using Complex = std::complex<FloatType>;
  using Buffer = b200vector<FloatType>;
  using ComplexBuffer = b200vector<Complex>;

  static constexpr bool handles_distributed = true;
  /// Unused when handles_distributed is true, required by the concept.
  static constexpr bool use_alltoallw = false;
  static constexpr bool use_p2p = false;

  struct DistributedInfo {
    int local_shape[D];
    int global_start[D];
    int output_shape[D];
    int output_start[D];
    std::size_t required_size;
  };

  explicit B200GridBackend(int num_stages, MPI_Comm comm,
                           FFTPlanFlag plan_flag = FFTPlanFlag::Estimate)
      : plan_flag_(plan_flag), comm_(comm) {
    (void)num_stages;
  }
  explicit B200GridBackend(int num_stages, FFTPlanFlag plan_flag = FFTPlanFlag::Estimate)
      : plan_flag_(plan_flag), comm_(MPI_COMM_WORLD) {
    (void)num_stages;
  }

  ~B200GridBackend() { release(); }
  B200GridBackend(const B200GridBackend &) = delete;
  B200GridBackend &operator=(const B200GridBackend &) = delete;
  B200GridBackend(B200GridBackend &&o) noexcept
      : plan_flag_(o.plan_flag_), comm_(o.comm_), shape_(o.shape_), info_(o.info_),
        cbuf_(std::move(o.cbuf_)), rbuf_(std::move(o.rbuf_)), copy_h_(o.copy_h_),
        ready_(o.ready_), c2c_built_(o.c2c_built_), real_built_(o.real_built_) {
    for (int t = 0; t < kTransforms; ++t) {
      h_[t] = o.h_[t];
      g_[t] = o.g_[t];
      o.h_[t] = nullptr;
      o.g_[t] = nullptr;
    }
    o.copy_h_ = nullptr;
    o.ready_ = false;
    o.c2c_built_ = o.real_built_ = false;
  }

  // ---- distributed part of the concept (fft_backend.hpp:153-190) ----------
  void setup_distributed(const int global_shape[D], MPI_Comm comm) {
    int size = 1;
    MPI_Comm_size(comm, &size);
    if (size != 1)
      throw std::runtime_error("B200GridBackend owns the grid on one GPU: communicator has " +
                               std::to_string(size) + " ranks");
    comm_ = comm;
    release();
    ready_ = false;
    long long n = 1;
    for (int i = 0; i < D; ++i) {
      if (global_shape[i] < 1)
        throw std::runtime_error("B200GridBackend: every extent must be >= 1");
      shape_[i] = global_shape[i];
      n *= global_shape[i];
      info_.local_shape[i] = info_.output_shape[i] = global_shape[i];
      info_.global_start[i] = info_.output_start[i] = 0;
    }
    info_.required_size = static_cast<std::size_t>(n);
    open(copy_h_, 1);
    ready_ = true;
  }

  DistributedInfo get_distributed_info() const { return info_; }

  Complex *get_buffer() {
    ensure_c2c();
    return cbuf_.data();
  }
  FloatType *get_real_buffer() {
    ensure_real();
    return rbuf_.data();
  }

  void forward() {
    ensure_c2c();
    run(kC2CForward);
  }
  void backward() {
    ensure_c2c();
    run(kC2CBackward);
  }
  void forward_r2c() {
    ensure_real();
    run(kR2C);
  }
  void backward_c2r() {
    ensure_real();
    run(kC2R);
  }

  // ---- the rest of the concept ----------------------------------------------
  void memcpy(void *dest, const void *src, std::size_t bytes) const {
    b200_detail::check(b200fft_memcpy(copy_h_, dest, src, bytes), "memcpy");
  }
  void memcpy2d(void *dst, std::size_t dpitch, const void *src, std::size_t spitch,
                std::size_t width, std::size_t height) const {
    b200_detail::check(b200fft_memcpy2d(copy_h_, dst, dpitch, src, spitch, width, height),
                       "memcpy2d");
  }
  void sync() const {
    if (copy_h_)
      b200_detail::check(b200fft_sync(copy_h_), "sync");
  }
  void first_touch(void *, std::size_t) const {}
  // Per-stage entry points: never called when handles_distributed is true.
  void create_stage_plan(int, int, std::size_t, Complex *, std::ptrdiff_t, std::ptrdiff_t) {}
  void execute_stage(int, FFTDirection, Complex *) {}
  void create_r2c_inplace_plan(int, std::size_t, FloatType *, std::ptrdiff_t, std::ptrdiff_t) {}
  void execute_r2c_inplace(FloatType *) {}
  void create_c2r_inplace_plan(int, std::size_t, FloatType *, std::ptrdiff_t, std::ptrdiff_t) {}
  void execute_c2r_inplace(FloatType *) {}

  // ---- extras ----------------------------------------------------------------
  /// The handle of one transform (0 C2C forward, 1 C2C backward, 2 R2C, 3 C2R).
  b200fft_handle handle(int transform) const { return h_[transform]; }
  /// Launches of one transform's recorded schedule (b200fft_group_stats).
  b200fft_stats schedule_stats(int transform) const {
    b200fft_stats s{};
    b200_detail::check(b200fft_group_stats(g_[transform], &s), "schedule stats");
    return s;
  }

private:
  enum { kC2CForward = 0, kC2CBackward = 1, kR2C = 2, kC2R = 3, kTransforms = 4 };

  // A side (C2C, or R2C with C2R) counts as built only once both of its
  // transforms are recorded and captured; if either build throws, the
  // handles and groups of that side are released so the next call starts
  // again from nothing.
  void ensure_c2c() {
    if (!ready_)
      throw std::runtime_error("B200GridBackend: setup_distributed was not called");
    if (c2c_built_)
      return;
    try {
      cbuf_.resize(info_.required_size);
      build_c2c(kC2CForward, B200FFT_FORWARD);
      build_c2c(kC2CBackward, B200FFT_BACKWARD);
    } catch (...) {
      release_transform(kC2CForward);
      release_transform(kC2CBackward);
      throw;
    }
    c2c_built_ = true;
  }
  void ensure_real() {
    if (!ready_)
      throw std::runtime_error("B200GridBackend: setup_distributed was not called");
    if (real_built_)
      return;
    try {
      const long long rows = static_cast<long long>(info_.required_size) / shape_[D - 1];
      rbuf_.resize(static_cast<std::size_t>(rows * 2 * (shape_[D - 1] / 2 + 1)));
      build_real(kR2C);
      build_real(kC2R);
    } catch (...) {
      release_transform(kR2C);
      release_transform(kC2R);
      throw;
    }
    real_built_ = true;
  }

  void open(b200fft_handle &h, int stages) {
    const int prec = std::is_same<FloatType, double>::value ? B200FFT_F64 : B200FFT_F32;
    const int pf = plan_flag_ == FFTPlanFlag::Estimate
                       ? B200FFT_PLAN_ESTIMATE
                       : (plan_flag_ == FFTPlanFlag::Measure ? B200FFT_PLAN_MEASURE
                                                             : B200FFT_PLAN_PATIENT);
    b200_detail::check(b200fft_create(prec, stages, pf, 0u, &h), "construct");
  }

  // C2C plan of axis k of a row-major grid `ext` (complex elements), stage k:
  // the last axis as rows, the others as columns over their trailing extent.
  void plan_axis(b200fft_handle h, const long long *ext, int naxes, int k, void *buf) {
    long long trailing = 1;
    for (int j = k + 1; j < naxes; ++j)
      trailing *= ext[j];
    long long total = 1;
    for (int j = 0; j < naxes; ++j)
      total *= ext[j];
    if (plan_flag_ != FFTPlanFlag::Estimate)
      b200_detail::check(b200fft_set_work_buffer(h, buf, 0), "planning buffer");
    if (k == naxes - 1)
      b200_detail::check(b200fft_plan_c2c(h, k, static_cast<int>(ext[k]),
                                          static_cast<std::size_t>(total / ext[k]), 1, ext[k]),
                         "plan (rows)");
    else
      b200_detail::check(b200fft_plan_c2c(h, k, static_cast<int>(ext[k]),
                                          static_cast<std::size_t>(trailing), trailing, 1),
                         "plan (columns)");
  }

  // The pass of axis k over the whole grid: one call for the first and last
  // axes, the slice loop (coalesced by the engine into one launch) otherwise.
  void exec_axis(b200fft_handle h, const long long *ext, int naxes, int k, int dir,
                 Complex *buf) {
    if (k == 0 || k == naxes - 1) {
      b200_detail::check(b200fft_exec_c2c(h, k, dir, buf), "pass");
      return;
    }
    long long lead = 1, slice = 1;
    for (int j = 0; j < k; ++j)
      lead *= ext[j];
    for (int j = k; j < naxes; ++j)
      slice *= ext[j];
    for (long long i = 0; i < lead; ++i)
      b200_detail::check(b200fft_exec_c2c(h, k, dir, buf + i * slice), "pass (slice)");
  }

  void record(int t) {
    b200_detail::check(b200fft_group_create(&g_[t]), "group");
    b200_detail::check(b200fft_group_add(g_[t], h_[t]), "group add");
    b200_detail::check(b200fft_group_begin(g_[t]), "group begin");
  }
  void capture(int t) {
    b200_detail::check(b200fft_group_end(g_[t]), "group end");
    b200_detail::check(b200fft_group_sync(g_[t]), "group sync");
    b200_detail::check(b200fft_group_capture(g_[t]), "graph capture");
  }

  void build_c2c(int t, int dir) {
    long long ext[D];
    for (int i = 0; i < D; ++i)
      ext[i] = shape_[i];
    open(h_[t], D);
    for (int k = 0; k < D; ++k)
      plan_axis(h_[t], ext, D, k, cbuf_.data());
    record(t);
    for (int s = 0; s < D; ++s) // forward: last axis first; backward: first axis first
      exec_axis(h_[t], ext, D, dir == B200FFT_FORWARD ? D - 1 - s : s, dir, cbuf_.data());
    capture(t);
  }

  void build_real(int t) {
    const long long n = shape_[D - 1];
    const long long nh = n / 2 + 1;
    long long ext[D]; // the complex view: [N0]...[N_{D-2}][N/2+1]
    long long rows = 1;
    for (int i = 0; i < D - 1; ++i) {
      ext[i] = shape_[i];
      rows *= shape_[i];
    }
    ext[D - 1] = nh;
    open(h_[t], D - 1);
    FloatType *real = rbuf_.data();
    Complex *cx = reinterpret_cast<Complex *>(real);
    if (plan_flag_ != FFTPlanFlag::Estimate)
      b200_detail::check(b200fft_set_work_buffer(h_[t], real, 0), "planning buffer");
    if (t == kR2C)
      b200_detail::check(b200fft_plan_r2c(h_[t], static_cast<int>(n),
                                          static_cast<std::size_t>(rows), 1, 2 * nh),
                         "plan (R2C rows)");
    else
      b200_detail::check(b200fft_plan_c2r(h_[t], static_cast<int>(n),
                                          static_cast<std::size_t>(rows), 1, 2 * nh),
                         "plan (C2R rows)");
    for (int k = 0; k < D - 1; ++k)
      plan_axis(h_[t], ext, D, k, real);
    record(t);
    if (t == kR2C) {
      b200_detail::check(b200fft_exec_r2c(h_[t], real), "R2C rows");
      for (int k = D - 2; k >= 0; --k)
        exec_axis(h_[t], ext, D, k, B200FFT_FORWARD, cx);
    } else {
      for (int k = 0; k <= D - 2; ++k)
        exec_axis(h_[t], ext, D, k, B200FFT_BACKWARD, cx);
      b200_detail::check(b200fft_exec_c2r(h_[t], real), "C2R rows");
    }
    capture(t);
  }

  void run(int t) {
    b200_detail::check(b200fft_group_replay(g_[t]), "replay");
    b200_detail::check(b200fft_group_sync(g_[t]), "wait");
  }

  void release_transform(int t) {
    if (g_[t])
      b200fft_group_destroy(g_[t]);
    if (h_[t])
      b200fft_destroy(h_[t]);
    g_[t] = nullptr;
    h_[t] = nullptr;
  }
  void release() {
    for (int t = 0; t < kTransforms; ++t)
      release_transform(t);
    c2c_built_ = real_built_ = false;
    if (copy_h_)
      b200fft_destroy(copy_h_);
    copy_h_ = nullptr;
  }

  FFTPlanFlag plan_flag_;
  MPI_Comm comm_;
  std::array<int, D> shape_{};
  DistributedInfo info_{};
  ComplexBuffer cbuf_;
  Buffer rbuf_;
  b200fft_handle h_[kTransforms] = {nullptr, nullptr, nullptr, nullptr};
  b200fft_group g_[kTransforms] = {nullptr, nullptr, nullptr, nullptr};
  b200fft_handle copy_h_ = nullptr;
  bool ready_ = false;      // setup_distributed has run
  bool c2c_built_ = false;  // both C2C transforms recorded and captured
  bool real_built_ = false; // R2C and C2R recorded and captured
};

} // namespace parafaft

#endif // PARAFAFT_BACKEND_B200_GRID_HPP
