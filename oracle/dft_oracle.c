/*
 * dft_oracle.c — FP64 CPU restatement of the transforms ParaFaFT delegates to
 * FFTW. TEST INFRASTRUCTURE ONLY: the parity checker of this repository, never
 * part of the product path.
 *
 * What it restates (FFTW 3, third-party, not vendored in ParaFaFT; version
 * unpinned there: cmake/fftw.cmake:1-45, cmake/parafaftConfig.cmake.in:8):
 *   - fftw_plan_guru64_dft with sign FFTW_FORWARD (-1) / FFTW_BACKWARD (+1),
 *     unnormalised (backend/fftw3/fft_backend_fftw.hpp:88-102, :419-422);
 *   - fftw_plan_guru64_dft_r2c: N reals -> N/2+1 complex (:465-467);
 *   - fftw_plan_guru64_dft_c2r: N/2+1 complex -> N reals, Hermitian input,
 *     imaginary parts of the DC and (even N) Nyquist terms ignored (:526-528).
 * The algorithm is the textbook mixed-radix decimation-in-time Cooley-Tukey
 * recursion: n = p*m with p the smallest prime factor, m-point transforms of
 * the p decimated subsequences, then p-point DFTs of the twiddled outputs.
 * Twiddles exp(-+2*pi*i*e/n) are evaluated in long double from an exactly
 * reduced integer exponent e mod n and rounded once to double.
 *
 * Batched n-D drivers transform every line along an axis of a row-major array
 * (OpenMP over lines), which is what ParaFaFT's per-axis stages compute on a
 * single rank.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cplx;

static long smallest_factor(long n) {
  if (n % 2 == 0)
    return 2;
  for (long p = 3; p * p <= n; p += 2)
    if (n % p == 0)
      return p;
  return n;
}

/* exp(sign*2*pi*i*e/n) for integer e, long double evaluation. */
static cplx twiddle(long e, long n, int sign) {
  e %= n;
  if (e < 0)
    e += n;
  const long double pi = 3.141592653589793238462643383279502884L;
  const long double a = 2.0L * pi * (long double)e / (long double)n;
  cplx w;
  w.re = (double)cosl(a);
  w.im = (double)(sign * sinl(a));
  return w;
}

/* out[k] = sum_j in[j*stride] exp(sign*2*pi*i*j*k/n), k < n (out contiguous). */
static void fft_rec(const cplx *in, long stride, cplx *out, long n, int sign,
                    const cplx *tw, long twn) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const long p = smallest_factor(n);
  const long m = n / p;
  /* sub-transforms of x[r + p*j] into out[r*m .. r*m+m) */
  for (long r = 0; r < p; ++r)
    fft_rec(in + r * stride, stride * p, out + r * m, m, sign, tw, twn);
  cplx *t = (cplx *)malloc(sizeof(cplx) * (size_t)p);
  cplx *y = (cplx *)malloc(sizeof(cplx) * (size_t)p);
  const long step = twn / n; /* tw has twn entries: tw[e] = exp(sign 2 pi i e/twn) */
  for (long k = 0; k < m; ++k) {
    for (long r = 0; r < p; ++r) {
      const cplx a = out[r * m + k];
      const cplx w = tw[((r * k) % n) * step];
      t[r].re = a.re * w.re - a.im * w.im;
      t[r].im = a.re * w.im + a.im * w.re;
    }
    for (long q = 0; q < p; ++q) {
      double sr = 0.0, si = 0.0;
      for (long r = 0; r < p; ++r) {
        const cplx w = tw[((r * q * m) % n) * step];
        sr += t[r].re * w.re - t[r].im * w.im;
        si += t[r].re * w.im + t[r].im * w.re;
      }
      y[q].re = sr;
      y[q].im = si;
    }
    for (long q = 0; q < p; ++q)
      out[k + q * m] = y[q];
  }
  free(t);
  free(y);
}

static cplx *make_table(long n, int sign) {
  cplx *tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  for (long e = 0; e < n; ++e)
    tw[e] = twiddle(e, n, sign);
  return tw;
}

/* One in-place 1D transform of n points at stride `stride` (complex units). */
void oracle_fft1d(double *data, long n, long stride, int sign) {
  cplx *x = (cplx *)data;
  cplx *in = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  cplx *out = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  cplx *tw = make_table(n, sign);
  for (long j = 0; j < n; ++j)
    in[j] = x[j * stride];
  fft_rec(in, 1, out, n, sign, tw, n);
  for (long j = 0; j < n; ++j)
    x[j * stride] = out[j];
  free(in);
  free(out);
  free(tw);
}

/* Batched strided 1D C2C, the semantics of a backend stage plan
 * (length, batch, stride, dist) executed in place. */
void oracle_c2c_batch(double *data, long length, long batch, long stride, long dist,
                      int sign) {
  cplx *tw = make_table(length, sign);
#pragma omp parallel
  {
    cplx *in = (cplx *)malloc(sizeof(cplx) * (size_t)length);
    cplx *out = (cplx *)malloc(sizeof(cplx) * (size_t)length);
#pragma omp for schedule(static)
    for (long b = 0; b < batch; ++b) {
      cplx *x = (cplx *)data + b * dist;
      for (long j = 0; j < length; ++j)
        in[j] = x[j * stride];
      fft_rec(in, 1, out, length, sign, tw, length);
      for (long j = 0; j < length; ++j)
        x[j * stride] = out[j];
    }
    free(in);
    free(out);
  }
  free(tw);
}

/* Batched R2C: n reals at real[b*idist + j*stride] -> n/2+1 complex at
 * cplx[b*odist + k*stride] (odist, stride in complex units). in and out may
 * alias (in-place padded layout): each row is read completely first. */
void oracle_r2c_batch(const double *real, double *outc, long n, long batch, long stride,
                      long idist, long odist) {
  cplx *tw = make_table(n, -1);
#pragma omp parallel
  {
    cplx *in = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    cplx *out = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for schedule(static)
    for (long b = 0; b < batch; ++b) {
      const double *x = real + b * idist;
      for (long j = 0; j < n; ++j) {
        in[j].re = x[j * stride];
        in[j].im = 0.0;
      }
      fft_rec(in, 1, out, n, -1, tw, n);
      cplx *y = (cplx *)outc + b * odist;
      for (long k = 0; k <= n / 2; ++k)
        y[k * stride] = out[k];
    }
    free(in);
    free(out);
  }
  free(tw);
}

/* Batched C2R (FFTW semantics, Im(DC) and Im(Nyquist) ignored). */
void oracle_c2r_batch(const double *inc, double *real, long n, long batch, long stride,
                      long idist, long odist) {
  cplx *tw = make_table(n, +1);
#pragma omp parallel
  {
    cplx *in = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    cplx *out = (cplx *)malloc(sizeof(cplx) * (size_t)n);
#pragma omp for schedule(static)
    for (long b = 0; b < batch; ++b) {
      const cplx *y = (const cplx *)inc + b * idist;
      for (long k = 0; k <= n / 2; ++k)
        in[k] = y[k * stride];
      in[0].im = 0.0;
      if (n % 2 == 0)
        in[n / 2].im = 0.0;
      for (long k = n / 2 + 1; k < n; ++k) {
        in[k].re = in[n - k].re;
        in[k].im = -in[n - k].im;
      }
      fft_rec(in, 1, out, n, +1, tw, n);
      double *x = real + b * odist;
      for (long j = 0; j < n; ++j)
        x[j * stride] = out[j].re;
    }
    free(in);
    free(out);
  }
  free(tw);
}

/* n-D C2C over a row-major array of `ndim` axes, every axis, in place. */
void oracle_c2c_nd(double *data, int ndim, const long *shape, int sign) {
  long total = 1;
  for (int d = 0; d < ndim; ++d)
    total *= shape[d];
  for (int ax = 0; ax < ndim; ++ax) {
    long inner = 1;
    for (int d = ax + 1; d < ndim; ++d)
      inner *= shape[d];
    const long n = shape[ax];
    const long outer = total / (n * inner);
    for (long o = 0; o < outer; ++o)
      oracle_c2c_batch(data + 2 * o * n * inner, n, inner, inner, 1, sign);
  }
}

/* Direct O(n^2) DFT in long double, for pinning the fast path on small n. */
void oracle_dft_direct(const double *in, double *out, long n, int sign) {
  const cplx *x = (const cplx *)in;
  cplx *y = (cplx *)out;
  const long double pi = 3.141592653589793238462643383279502884L;
  for (long k = 0; k < n; ++k) {
    long double sr = 0.0L, si = 0.0L;
    for (long j = 0; j < n; ++j) {
      const long e = (j * k) % n;
      const long double a = 2.0L * pi * (long double)e / (long double)n;
      const long double c = cosl(a), s = sign * sinl(a);
      sr += x[j].re * c - x[j].im * s;
      si += x[j].re * s + x[j].im * c;
    }
    y[k].re = (double)sr;
    y[k].im = (double)si;
  }
}
