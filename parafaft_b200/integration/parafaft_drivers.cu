// ParaFaFT's own orchestrators, ParaFaFT_C2C<D, Backend> and
// ParaFaFT_R2C<D, Backend> (parafaft_c2c.hpp:69, parafaft_r2c.hpp:98),
// instantiated with B200Backend<T> — the drop-in this project provides — and
// B200GridBackend<D, T> (its grid-owning form), and, for comparison on the
// same GPU, with the reference CuFFTBackend<T>
// (backend/cufft/fft_backend_cufft.hpp). A small C ABI exposes the objects to
// the Python tests and the benchmark, so every transform they run goes through
// the reference's forward()/backward() code path unchanged.
//
// Built only where the ParaFaFT headers are present. FFTW is not installed
// here, so the FFTW backend header is skipped; ParaFaFT only names
// FFTWBackend<> as a default template argument, which a declaration
// satisfies.
#define PARAFAFT_BACKEND_FFTW_HPP 1
namespace parafaft {
template <typename FloatTypeT = double> class FFTWBackend;
}
// The product build (libparafaft_b200_drivers.so) leaves the reference's
// cuFFT backend out, so it does not link cuFFT; the comparator build
// (libparafaft_cufft_drivers.so, compiled with PFB_WITH_CUFFT) adds it.
#ifndef PFB_WITH_CUFFT
#define PARAFAFT_BACKEND_CUFFT_HPP 1
#endif

#include <mpi.h>

#include <memory>
#include <stdexcept>
#include <string>

#include "parafaft_c2c.hpp"
#include "parafaft_r2c.hpp"

#include "b200fft.h"
#include "fft_backend_b200.hpp"
#include "fft_backend_b200_grid.hpp"

namespace {

thread_local std::string g_err;

struct Obj {
  virtual ~Obj() = default;
  virtual void forward(void *data) = 0;
  virtual void backward(void *data) = 0;
  virtual void forward_oop(const void *in, void *out) = 0;
  virtual void backward_oop(void *in, void *out) = 0;
  virtual long long required_size() const = 0;
  virtual void shapes(int *in_shape, int *in_start, int *out_shape, int *out_start) const = 0;
  // the backend-owned grid buffer (backends with handles_distributed), else null
  virtual void *buffer() { return nullptr; }
  int ndim = 0;
  bool r2c = false;
  b200fft_handle handle = nullptr;
};

template <int D, class B> struct C2CObj : Obj {
  using F = parafaft::ParaFaFT_C2C<D, B>;
  using Cx = typename B::Complex;
  std::unique_ptr<F> f;
  C2CObj(const int *shape, parafaft::FFTPlanFlag flag) {
    parafaft::b200_detail::last_opened() = nullptr;
    f.reset(new F(shape, MPI_COMM_WORLD, flag));
    handle = parafaft::b200_detail::last_opened();
    this->ndim = D;
  }
  void forward(void *d) override { f->forward(static_cast<Cx *>(d)); }
  void backward(void *d) override { f->backward(static_cast<Cx *>(d)); }
  void forward_oop(const void *, void *) override {
    throw std::runtime_error("out-of-place transforms exist for R2C objects only");
  }
  void backward_oop(void *, void *) override {
    throw std::runtime_error("out-of-place transforms exist for R2C objects only");
  }
  long long required_size() const override {
    return static_cast<long long>(f->get_required_output_size());
  }
  void *buffer() override { return f->get_buffer(); }
  void shapes(int *a, int *b, int *c, int *d) const override {
    f->get_local_shape(a);
    f->get_global_start(b);
    f->get_final_shape(c);
    f->get_final_start(d);
  }
};

template <int D, class B> struct R2CObj : Obj {
  using F = parafaft::ParaFaFT_R2C<D, B>;
  using Cx = typename B::Complex;
  using Fl = typename B::FloatType;
  std::unique_ptr<F> f;
  R2CObj(const int *shape, parafaft::FFTPlanFlag flag) {
    parafaft::b200_detail::last_opened() = nullptr;
    f.reset(new F(shape, MPI_COMM_WORLD, flag));
    handle = parafaft::b200_detail::last_opened();
    this->ndim = D;
    this->r2c = true;
  }
  void forward(void *d) override { f->forward_in_place(static_cast<Fl *>(d)); }
  void backward(void *d) override { f->backward_in_place(static_cast<Fl *>(d)); }
  void forward_oop(const void *in, void *out) override {
    f->forward(static_cast<const Fl *>(in), static_cast<Cx *>(out));
  }
  void backward_oop(void *in, void *out) override {
    f->backward(static_cast<Cx *>(in), static_cast<Fl *>(out));
  }
  long long required_size() const override {
    return static_cast<long long>(f->get_required_output_size());
  }
  void *buffer() override { return f->get_real_buffer(); }
  void shapes(int *a, int *b, int *c, int *d) const override {
    f->get_local_real_shape(a);
    f->get_real_global_start(b);
    f->get_local_complex_shape(c);
    f->get_complex_global_start(d);
  }
};

// One-rank C2C transform driving a backend with the same call sequence as
// ParaFaFT_C2C::forward/backward on one rank (parafaft_c2c.hpp:539-694):
// plans per stage (last axis contiguous, first axis strided, middle axes one
// slab per leading index, :249-287), a copy into the scratch buffer first when
// D-1 is odd, then per stage the transform followed by the one-rank exchange
// (a full-buffer copy, parafaft_common.hpp:488-494), ending in sync(). On one
// rank every stage buffer has the global shape; ParaFaFT_C2C instead sizes
// redistributed axes from another axis' extent (parafaft_c2c.hpp:826-831),
// which is only right for hypercubic grids, so non-hypercubic grids are run
// through this object.
template <class B> b200fft_handle handle_of(const B &) { return nullptr; }
template <class T> b200fft_handle handle_of(const parafaft::B200Backend<T> &b) {
  return b.handle();
}

template <int D, class B> struct OneRankC2C : Obj {
  using Cx = typename B::Complex;
  B backend;
  int shape[D];
  std::size_t total = 1;
  typename B::ComplexBuffer scratch;
  OneRankC2C(const int *s, parafaft::FFTPlanFlag flag) : backend(D, flag) {
    handle = handle_of(backend);
    this->ndim = D;
    for (int i = 0; i < D; ++i) {
      shape[i] = s[i];
      total *= static_cast<std::size_t>(s[i]);
    }
    scratch.resize(total);
    for (int stage = 0; stage < D; ++stage) {
      const int axis = D - 1 - stage;
      const std::size_t n = static_cast<std::size_t>(shape[axis]);
      std::size_t trailing = 1;
      for (int i = axis + 1; i < D; ++i)
        trailing *= static_cast<std::size_t>(shape[i]);
      if (axis == D - 1)
        backend.create_stage_plan(stage, shape[axis], total / n, scratch.data(), 1,
                                  static_cast<std::ptrdiff_t>(n));
      else if (axis == 0)
        backend.create_stage_plan(stage, shape[axis], total / n, scratch.data(),
                                  static_cast<std::ptrdiff_t>(total / n), 1);
      else
        backend.create_stage_plan(stage, shape[axis], trailing, scratch.data(),
                                  static_cast<std::ptrdiff_t>(trailing), 1);
    }
  }
  void stage_fft(int stage, parafaft::FFTDirection dir, Cx *buf) {
    const int axis = D - 1 - stage;
    if (axis == 0 || axis == D - 1) {
      backend.execute_stage(stage, dir, buf);
      return;
    }
    std::size_t leading = 1, slab = static_cast<std::size_t>(shape[axis]);
    for (int i = 0; i < axis; ++i)
      leading *= static_cast<std::size_t>(shape[i]);
    for (int i = axis + 1; i < D; ++i)
      slab *= static_cast<std::size_t>(shape[i]);
    for (std::size_t i = 0; i < leading; ++i)
      backend.execute_stage(stage, dir, buf + i * slab);
  }
  void run(Cx *data, bool fwd) {
    Cx *src = data, *dst = scratch.data();
    if ((D - 1) % 2 != 0) {
      backend.memcpy(scratch.data(), data, total * sizeof(Cx));
      src = scratch.data();
      dst = data;
    }
    const auto dir = fwd ? parafaft::FFTDirection::Forward : parafaft::FFTDirection::Backward;
    for (int k = 0; k < D; ++k) {
      const int stage = fwd ? k : D - 1 - k;
      stage_fft(stage, dir, src);
      if (k < D - 1) {
        backend.memcpy(dst, src, total * sizeof(Cx));
        std::swap(src, dst);
      }
    }
    backend.sync();
  }
  void forward(void *d) override { run(static_cast<Cx *>(d), true); }
  void backward(void *d) override { run(static_cast<Cx *>(d), false); }
  void forward_oop(const void *, void *) override {
    throw std::runtime_error("out-of-place transforms exist for R2C objects only");
  }
  void backward_oop(void *, void *) override {
    throw std::runtime_error("out-of-place transforms exist for R2C objects only");
  }
  long long required_size() const override { return static_cast<long long>(total); }
  void shapes(int *a, int *b, int *c, int *d) const override {
    for (int i = 0; i < D; ++i) {
      a[i] = c[i] = shape[i];
      b[i] = d[i] = 0;
    }
  }
};

template <template <int, class> class O, class B>
Obj *make_d(int D, const int *shape, parafaft::FFTPlanFlag flag) {
  switch (D) {
  case 2: return new O<2, B>(shape, flag);
  case 3: return new O<3, B>(shape, flag);
  case 4: return new O<4, B>(shape, flag);
  case 5: return new O<5, B>(shape, flag);
  default: throw std::runtime_error("D must be 2..5");
  }
}

template <template <int, class> class O>
Obj *make(int D, int prec, int backend, const int *shape, int plan_flag) {
  const auto flag = static_cast<parafaft::FFTPlanFlag>(plan_flag);
  if (backend == 0)
    return prec == B200FFT_F64 ? make_d<O, parafaft::B200Backend<double>>(D, shape, flag)
                               : make_d<O, parafaft::B200Backend<float>>(D, shape, flag);
#ifdef PFB_WITH_CUFFT
  if (backend == 1)
    return prec == B200FFT_F64 ? make_d<O, parafaft::CuFFTBackend<double>>(D, shape, flag)
                               : make_d<O, parafaft::CuFFTBackend<float>>(D, shape, flag);
#else
  if (backend == 1)
    throw std::runtime_error("CuFFTBackend objects live in libparafaft_cufft_drivers.so");
#endif
  throw std::runtime_error("backend must be 0 (B200Backend) or 1 (CuFFTBackend)");
}

// ParaFaFT objects on B200GridBackend<D, T> (the grid-owning backend; the
// reference orchestrators only, whose distributed path takes any shape).
template <template <int, class> class O, class T>
Obj *make_grid_t(int D, const int *shape, parafaft::FFTPlanFlag flag) {
  switch (D) {
  case 2: return new O<2, parafaft::B200GridBackend<2, T>>(shape, flag);
  case 3: return new O<3, parafaft::B200GridBackend<3, T>>(shape, flag);
  case 4: return new O<4, parafaft::B200GridBackend<4, T>>(shape, flag);
  case 5: return new O<5, parafaft::B200GridBackend<5, T>>(shape, flag);
  default: throw std::runtime_error("D must be 2..5");
  }
}
template <template <int, class> class O>
Obj *make_grid(int D, int prec, const int *shape, int plan_flag) {
  const auto flag = static_cast<parafaft::FFTPlanFlag>(plan_flag);
  return prec == B200FFT_F64 ? make_grid_t<O, double>(D, shape, flag)
                             : make_grid_t<O, float>(D, shape, flag);
}

template <class F> int guard(F f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  } catch (...) {
    g_err = "unknown exception";
    return -1;
  }
}

} // namespace

extern "C" {

const char *pfb_last_error(void) { return g_err.c_str(); }

// kind: 0 C2C (ParaFaFT_C2C), 1 R2C (ParaFaFT_R2C), 2 C2C through the
// one-rank orchestrator above (any grid shape). backend: 0 B200Backend,
// 1 CuFFTBackend, 2 B200GridBackend (the grid-owning backend: kinds 0 and 1;
// forward/backward then ignore their data argument and transform the buffer
// pfb_buffer returns). prec: B200FFT_F32/F64.
int pfb_create(int kind, int D, int prec, int backend, const int *shape, int plan_flag,
               void **out) {
  return guard([&] {
    *out = nullptr;
    if (backend == 2 && kind == 2)
      throw std::runtime_error("the grid-owning backend runs through the reference "
                               "orchestrators (kind c2c or r2c)");
    Obj *o = backend == 2 ? (kind == 0 ? make_grid<C2CObj>(D, prec, shape, plan_flag)
                                       : make_grid<R2CObj>(D, prec, shape, plan_flag))
             : kind == 0  ? make<C2CObj>(D, prec, backend, shape, plan_flag)
             : kind == 1  ? make<R2CObj>(D, prec, backend, shape, plan_flag)
                          : make<OneRankC2C>(D, prec, backend, shape, plan_flag);
    *out = o;
  });
}

int pfb_destroy(void *h) {
  return guard([&] { delete static_cast<Obj *>(h); });
}

int pfb_forward(void *h, void *data) {
  return guard([&] { static_cast<Obj *>(h)->forward(data); });
}

int pfb_backward(void *h, void *data) {
  return guard([&] { static_cast<Obj *>(h)->backward(data); });
}

int pfb_forward_oop(void *h, const void *in, void *out) {
  return guard([&] { static_cast<Obj *>(h)->forward_oop(in, out); });
}

int pfb_backward_oop(void *h, void *in, void *out) {
  return guard([&] { static_cast<Obj *>(h)->backward_oop(in, out); });
}

long long pfb_required_size(void *h) { return static_cast<Obj *>(h)->required_size(); }

int pfb_shapes(void *h, int *in_shape, int *in_start, int *out_shape, int *out_start) {
  return guard([&] { static_cast<Obj *>(h)->shapes(in_shape, in_start, out_shape, out_start); });
}

// The B200 handle inside the object (null for CuFFTBackend objects).
void *pfb_b200_handle(void *h) { return static_cast<Obj *>(h)->handle; }
// Device pointer of the grid a grid-owning backend holds (null otherwise).
void *pfb_buffer(void *h) { return static_cast<Obj *>(h)->buffer(); }

} // extern "C"
