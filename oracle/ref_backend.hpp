// OracleBackend: a CPU backend for ParaFaFT's orchestrators whose 1D
// transforms are the FP64 oracle of dft_oracle.c. TEST INFRASTRUCTURE ONLY:
// it lets the reference's own ParaFaFT_C2C / ParaFaFT_R2C code (stage shapes,
// plans, ping-pong buffers, exchange calls) run on the CPU here, so golden
// fixtures come out of the reference's orchestration code.
//
// Mirrors FFTWBackend (backend/fftw3/fft_backend_fftw.hpp): host buffers,
// use_alltoallw = true (:586) so every stage transition goes through
// MPI_Alltoallw as it does with FFTW, in-place padded R2C/C2R with dist in
// reals and dist/2 complex on the complex side (:439-549).
#pragma once

#include <complex>
#include <cstddef>
#include <cstring>
#include <mpi.h>
#include <vector>

extern "C" {
void oracle_c2c_batch(double *data, long length, long batch, long stride, long dist, int sign);
void oracle_r2c_batch(const double *real, double *outc, long n, long batch, long stride,
                      long idist, long odist);
void oracle_c2r_batch(const double *inc, double *real, long n, long batch, long stride,
                      long idist, long odist);
}

namespace parafaft {

template <typename T> class OracleVector {
public:
  void resize(std::size_t n) { v_.assign(n, T()); }
  T *data() { return v_.data(); }
  const T *data() const { return v_.data(); }
  std::size_t size() const { return v_.size(); }

private:
  std::vector<T> v_;
};

template <typename FloatTypeT = double> class OracleBackend {
  static_assert(sizeof(FloatTypeT) == 8, "the oracle computes in double");

public:
  using FloatType = double;
  using Complex = std::complex<double>;
  using Buffer = OracleVector<double>;
  using ComplexBuffer = OracleVector<Complex>;
  static constexpr bool use_alltoallw = true;
  static constexpr bool handles_distributed = false;
  static constexpr bool use_p2p = false;

  explicit OracleBackend(int num_stages, FFTPlanFlag = FFTPlanFlag::Estimate)
      : plans_(num_stages) {}
  OracleBackend(int num_stages, MPI_Comm, FFTPlanFlag = FFTPlanFlag::Estimate)
      : plans_(num_stages) {}

  void create_stage_plan(int stage, int length, std::size_t batch, Complex *,
                         std::ptrdiff_t stride, std::ptrdiff_t dist) {
    plans_[stage] = {length, static_cast<long>(batch), static_cast<long>(stride),
                     static_cast<long>(dist)};
  }
  void execute_stage(int stage, FFTDirection dir, Complex *data) {
    const P &p = plans_[stage];
    oracle_c2c_batch(reinterpret_cast<double *>(data), p.n, p.batch, p.stride, p.dist,
                     dir == FFTDirection::Forward ? -1 : +1);
  }
  void create_r2c_inplace_plan(int n, std::size_t batch, double *, std::ptrdiff_t stride,
                               std::ptrdiff_t dist) {
    r2c_ = {n, static_cast<long>(batch), static_cast<long>(stride), static_cast<long>(dist)};
  }
  void execute_r2c_inplace(double *p) {
    oracle_r2c_batch(p, p, r2c_.n, r2c_.batch, r2c_.stride, r2c_.dist, r2c_.dist / 2);
  }
  void create_c2r_inplace_plan(int n, std::size_t batch, double *, std::ptrdiff_t stride,
                               std::ptrdiff_t dist) {
    c2r_ = {n, static_cast<long>(batch), static_cast<long>(stride), static_cast<long>(dist)};
  }
  void execute_c2r_inplace(double *p) {
    oracle_c2r_batch(p, p, c2r_.n, c2r_.batch, c2r_.stride, c2r_.dist / 2, c2r_.dist);
  }
  void memcpy(void *d, const void *s, std::size_t n) const { std::memmove(d, s, n); }
  void memcpy2d(void *dst, std::size_t dpitch, const void *src, std::size_t spitch,
                std::size_t width, std::size_t height) const {
    for (std::size_t r = 0; r < height; ++r)
      std::memmove(static_cast<char *>(dst) + r * dpitch,
                   static_cast<const char *>(src) + r * spitch, width);
  }
  void sync() const {}
  void first_touch(void *, std::size_t) const {}

private:
  struct P {
    int n;
    long batch, stride, dist;
  };
  std::vector<P> plans_;
  P r2c_{}, c2r_{};
};

} // namespace parafaft
