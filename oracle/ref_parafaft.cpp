// The reference's ParaFaFT_C2C / ParaFaFT_R2C orchestrators, compiled from the
// reference sources with the single-rank MPI stand-in and OracleBackend.
// TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref_parafaft.so); the golden
// fixture generator and the oracle's own tests call it.
#define PARAFAFT_BACKEND_FFTW_HPP 1
namespace parafaft {
template <typename FloatTypeT = double> class FFTWBackend;
}
#include <mpi.h>

#include <memory>
#include <stdexcept>
#include <string>

#include "parafaft_c2c.hpp"
#include "parafaft_r2c.hpp"
#include "ref_backend.hpp"

namespace {
thread_local std::string g_err;
struct Obj {
  virtual ~Obj() = default;
  virtual void fwd(void *) = 0;
  virtual void bwd(void *) = 0;
  virtual void fwd_oop(const void *, void *) = 0;
  virtual void bwd_oop(void *, void *) = 0;
  virtual long long req() const = 0;
  virtual void shapes(int *, int *, int *, int *) const = 0;
};
using B = parafaft::OracleBackend<double>;
template <int D> struct C2C : Obj {
  parafaft::ParaFaFT_C2C<D, B> f;
  explicit C2C(const int *s) : f(s, MPI_COMM_WORLD) {}
  void fwd(void *d) override { f.forward(static_cast<B::Complex *>(d)); }
  void bwd(void *d) override { f.backward(static_cast<B::Complex *>(d)); }
  void fwd_oop(const void *, void *) override { throw std::runtime_error("c2c has no oop"); }
  void bwd_oop(void *, void *) override { throw std::runtime_error("c2c has no oop"); }
  long long req() const override { return (long long)f.get_required_output_size(); }
  void shapes(int *a, int *b, int *c, int *d) const override {
    f.get_local_shape(a); f.get_global_start(b); f.get_final_shape(c); f.get_final_start(d);
  }
};
template <int D> struct R2C : Obj {
  parafaft::ParaFaFT_R2C<D, B> f;
  explicit R2C(const int *s) : f(s, MPI_COMM_WORLD) {}
  void fwd(void *d) override { f.forward_in_place(static_cast<double *>(d)); }
  void bwd(void *d) override { f.backward_in_place(static_cast<double *>(d)); }
  void fwd_oop(const void *i, void *o) override {
    f.forward(static_cast<const double *>(i), static_cast<B::Complex *>(o));
  }
  void bwd_oop(void *i, void *o) override {
    f.backward(static_cast<B::Complex *>(i), static_cast<double *>(o));
  }
  long long req() const override { return (long long)f.get_required_output_size(); }
  void shapes(int *a, int *b, int *c, int *d) const override {
    f.get_local_real_shape(a); f.get_real_global_start(b);
    f.get_local_complex_shape(c); f.get_complex_global_start(d);
  }
};
template <template <int> class O> Obj *make(int D, const int *s) {
  switch (D) {
  case 2: return new O<2>(s);
  case 3: return new O<3>(s);
  case 4: return new O<4>(s);
  case 5: return new O<5>(s);
  default: throw std::runtime_error("D must be 2..5");
  }
}
template <class F> int guard(F f) {
  try { f(); return 0; } catch (const std::exception &e) { g_err = e.what(); return -1; }
}
} // namespace

extern "C" {
const char *ref_last_error(void) { return g_err.c_str(); }
int ref_create(int kind, int D, const int *shape, void **out) {
  return guard([&] { *out = kind == 0 ? make<C2C>(D, shape) : make<R2C>(D, shape); });
}
int ref_destroy(void *h) { return guard([&] { delete static_cast<Obj *>(h); }); }
int ref_forward(void *h, void *d) { return guard([&] { static_cast<Obj *>(h)->fwd(d); }); }
int ref_backward(void *h, void *d) { return guard([&] { static_cast<Obj *>(h)->bwd(d); }); }
int ref_forward_oop(void *h, const void *i, void *o) {
  return guard([&] { static_cast<Obj *>(h)->fwd_oop(i, o); });
}
int ref_backward_oop(void *h, void *i, void *o) {
  return guard([&] { static_cast<Obj *>(h)->bwd_oop(i, o); });
}
long long ref_required_size(void *h) { return static_cast<Obj *>(h)->req(); }
int ref_shapes(void *h, int *a, int *b, int *c, int *d) {
  return guard([&] { static_cast<Obj *>(h)->shapes(a, b, c, d); });
}
}
