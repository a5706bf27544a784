// Device code of the B200 transform engine.
//
// Every transform is a Stockham autosort FFT over shared memory:
//   stage s, radix R, Ns = product of earlier radices, butterfly j < L/R:
//     read   x_r = a[j + r*L/R]                       (r < R)
//     twiddle x_r *= w^(r*(j mod Ns)),  w = exp(-+2*pi*i/(Ns*R))
//     DFT_R over (x_0..x_{R-1})
//     write  b[(j/Ns)*Ns*R + (j mod Ns) + r*Ns] = X_r
// The first stage reads global memory directly and the last stage writes it
// directly (its write index reduces to j + r*L/R), so a transform costs one
// HBM read and one HBM write plus (stages-1) shared-memory exchanges.
// Twiddles come from a table exp(-2*pi*i*m/tlen) generated once per length in
// FP64 by sincospi after exact integer reduction of m (twiddle_table_kernel),
// then rounded to the working precision.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_common.hpp"

namespace b200fft {

#define BF_D __device__ __forceinline__

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };
template <typename T> using cvec = typename Vec2<T>::type;

BF_D float2 cmake(float x, float y) { return make_float2(x, y); }
BF_D double2 cmake(double x, double y) { return make_double2(x, y); }
template <typename V> BF_D V czero() { V r; r.x = 0; r.y = 0; return r; }
template <typename V> BF_D V cadd(V a, V b) { return cmake(a.x + b.x, a.y + b.y); }
template <typename V> BF_D V csub(V a, V b) { return cmake(a.x - b.x, a.y - b.y); }
template <typename V> BF_D V cconj(V a) { return cmake(a.x, -a.y); }
// a * w, or a * conj(w) when CONJ
template <bool CONJ, typename V> BF_D V cmulw(V a, V w) {
  if (CONJ)
    return cmake(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
  return cmake(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
// multiply by -i (forward) or +i (backward)
template <bool FWD, typename V> BF_D V rot(V a) {
  return FWD ? cmake(a.y, -a.x) : cmake(-a.y, a.x);
}

BF_D uint32_t fdiv(uint32_t n, const FastDiv &f) {
  return f.m == 0 ? n : (__umulhi(n, f.m) >> f.s);
}

// Slab sl and position w of transform b < a.total (b = sl*batch + w). One
// slab (the common case, the same for the whole grid) needs no division;
// otherwise a 32-bit division when the transforms fit, else 64-bit (a 64-bit
// division is a long software sequence per warp).
BF_D void slab_of(const PassArgs &a, long long b, long long &sl, long long &w) {
  if (a.total == a.batch) {
    sl = 0;
    w = b;
  } else if (a.total <= 0xffffffffll) {
    const unsigned q = static_cast<unsigned>(b) / static_cast<unsigned>(a.batch);
    sl = q;
    w = b - static_cast<long long>(q) * a.batch;
  } else {
    sl = b / a.batch;
    w = b - sl * a.batch;
  }
}

// ---- small DFTs (natural order in and out) -------------------------------
template <bool FWD, typename V> BF_D void dft2(V &a, V &b) {
  V t = csub(a, b);
  a = cadd(a, b);
  b = t;
}

template <bool FWD, typename V> BF_D void dft3(V *v) {
  using T = decltype(v[0].x);
  const T s = T(0.86602540378443864676372317075294);
  V t = cadd(v[1], v[2]);
  V d = csub(v[1], v[2]);
  V m = cmake(v[0].x - T(0.5) * t.x, v[0].y - T(0.5) * t.y);
  V sd = rot<FWD>(cmake(s * d.x, s * d.y)); // -+ i*s*d
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, sd);
  v[2] = csub(m, sd);
}

template <bool FWD, typename V> BF_D void dft4(V &a0, V &a1, V &a2, V &a3) {
  V t0 = cadd(a0, a2), t1 = csub(a0, a2);
  V t2 = cadd(a1, a3), t3 = rot<FWD>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <bool FWD, typename V> BF_D void dft5(V *v) {
  using T = decltype(v[0].x);
  const T c1 = T(0.30901699437494742410229341718282);
  const T c2 = T(-0.80901699437494742410229341718282);
  const T s1 = T(0.95105651629515357211643933337938);
  const T s2 = T(0.58778525229247312916870595463907);
  V a = cadd(v[1], v[4]), b = csub(v[1], v[4]);
  V c = cadd(v[2], v[3]), d = csub(v[2], v[3]);
  V m1 = cmake(v[0].x + c1 * a.x + c2 * c.x, v[0].y + c1 * a.y + c2 * c.y);
  V m2 = cmake(v[0].x + c2 * a.x + c1 * c.x, v[0].y + c2 * a.y + c1 * c.y);
  V n1 = rot<FWD>(cmake(s1 * b.x + s2 * d.x, s1 * b.y + s2 * d.y));
  V n2 = rot<FWD>(cmake(s2 * b.x - s1 * d.x, s2 * b.y - s1 * d.y));
  v[0] = cmake(v[0].x + a.x + c.x, v[0].y + a.y + c.y);
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <bool FWD, typename V> BF_D void dft8(V *v) {
  using T = decltype(v[0].x);
  const T h = T(0.70710678118654752440084436210485);
  V e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  V o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<FWD>(e0, e1, e2, e3);
  dft4<FWD>(o0, o1, o2, o3);
  // o_k *= w8^k, w8 = exp(-+ i*pi/4)
  if (FWD) {
    o1 = cmake(h * (o1.x + o1.y), h * (o1.y - o1.x));
    o3 = cmake(h * (o3.y - o3.x), -h * (o3.x + o3.y));
  } else {
    o1 = cmake(h * (o1.x - o1.y), h * (o1.x + o1.y));
    o3 = cmake(-h * (o3.x + o3.y), h * (o3.x - o3.y));
  }
  o2 = rot<FWD>(o2);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// ---- 16- and 32-point butterflies from 4- and 8-point ones ---------------
// cos and sin of 2*pi*m/n at compile time: the angle is folded by symmetry
// into [0, pi/4] with exact integer arithmetic (in units of 1/(8n) turn), then
// summed from the Taylor series (16 terms: far below double rounding there).
struct CosSin {
  double c, s;
};
constexpr CosSin ce_cossin(long long m, long long n) {
  m %= n;
  if (m < 0)
    m += n;
  long long a = 8 * m, d = 8 * n; // angle = 2*pi*a/d
  bool neg_s = false, neg_c = false, swap = false;
  if (2 * a > d) { // 2*pi - x
    a = d - a;
    neg_s = true;
  }
  if (4 * a > d) { // pi - x
    a = d / 2 - a;
    neg_c = true;
  }
  if (8 * a > d) { // pi/2 - x
    a = d / 4 - a;
    swap = true;
  }
  const double x = 2.0 * 3.14159265358979323846264338327950288 * static_cast<double>(a) /
                   static_cast<double>(d);
  double ts = x, ss = x, tc = 1.0, sc = 1.0;
  for (int k = 1; k < 16; ++k) {
    ts *= -x * x / static_cast<double>((2 * k) * (2 * k + 1));
    tc *= -x * x / static_cast<double>((2 * k - 1) * (2 * k));
    ss += ts;
    sc += tc;
  }
  double c = swap ? ss : sc, sn = swap ? sc : ss;
  return CosSin{neg_c ? -c : c, neg_s ? -sn : sn};
}
template <int M, int N> struct TwC {
  static constexpr double c = ce_cossin(M, N).c;
  static constexpr double s = ce_cossin(M, N).s;
};

// a * exp(-+2*pi*i*M/N) for compile-time M, N (forward: minus). Multiples of
// an eighth of a turn cost at most two multiplications.
template <int M, int N, bool FWD, typename V> BF_D V twk(V a) {
  using T = decltype(a.x);
  constexpr int m = ((M % N) + N) % N;
  constexpr T h = T(0.70710678118654752440084436210485);
  if constexpr (m == 0) {
    return a;
  } else if constexpr (4 * m == N) {
    return rot<FWD>(a);
  } else if constexpr (2 * m == N) {
    return cmake(-a.x, -a.y);
  } else if constexpr (4 * m == 3 * N) {
    return rot<!FWD>(a);
  } else if constexpr (8 * m == N || 8 * m == 5 * N) {
    const V b = FWD ? cmake(h * (a.x + a.y), h * (a.y - a.x))
                    : cmake(h * (a.x - a.y), h * (a.x + a.y));
    return 8 * m == N ? b : cmake(-b.x, -b.y);
  } else if constexpr (8 * m == 3 * N || 8 * m == 7 * N) {
    const V b = FWD ? cmake(h * (a.y - a.x), -h * (a.x + a.y))
                    : cmake(-h * (a.x + a.y), h * (a.x - a.y));
    return 8 * m == 3 * N ? b : cmake(-b.x, -b.y);
  } else {
    constexpr T c = T(TwC<m, N>::c), sn = T(TwC<m, N>::s);
    return FWD ? cmake(a.x * c + a.y * sn, a.y * c - a.x * sn)
               : cmake(a.x * c - a.y * sn, a.y * c + a.x * sn);
  }
}

template <int R, bool FWD, typename V> BF_D void dft(V *v);

// N = N1*N2 points in natural order: n = N2*n1 + n2, k = k1 + N1*k2;
// N2 DFTs of N1 points over n1, the twiddles w_N^(n2*k1), then N1 DFTs of
// N2 points over n2.
template <int N1, int N2, bool FWD, typename V> struct CompositeDft {
  static constexpr int N = N1 * N2;
  template <int n2, int k1> static BF_D void twiddle_into(const V *u, V *t) {
    if constexpr (k1 < N1) {
      t[k1 * N2 + n2] = twk<n2 * k1, N, FWD>(u[k1]);
      twiddle_into<n2, k1 + 1>(u, t);
    }
  }
  template <int n2> static BF_D void inner(const V *v, V *t) {
    if constexpr (n2 < N2) {
      V u[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1)
        u[n1] = v[N2 * n1 + n2];
      dft<N1, FWD>(u);
      twiddle_into<n2, 0>(u, t);
      inner<n2 + 1>(v, t);
    }
  }
  static BF_D void run(V *v) {
    V t[N];
    inner<0>(v, t);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      dft<N2, FWD>(&t[k1 * N2]);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2)
        v[k1 + N1 * k2] = t[k1 * N2 + k2];
    }
  }
};

template <int R, bool FWD, typename V> BF_D void dft(V *v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<FWD>(v[0], v[1]);
  } else if constexpr (R == 3) {
    dft3<FWD>(v);
  } else if constexpr (R == 4) {
    dft4<FWD>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    dft5<FWD>(v);
  } else if constexpr (R == 8) {
    dft8<FWD>(v);
  } else if constexpr (R == 16) {
    CompositeDft<4, 4, FWD, V>::run(v);
  } else if constexpr (R == 32) {
    CompositeDft<4, 8, FWD, V>::run(v);
  } else {
    static_assert(R == 0, "unsupported radix");
  }
}

template <typename V> BF_D V ldtw(const V *tw, int m) { return __ldg(tw + m); }

// Asynchronous global->shared copies (cp.async): the data goes to shared
// memory without passing through registers; a commit group per tile lets a CTA
// wait for one tile while the next is still in flight.
template <typename V> BF_D void cp_async_elem(V *smem, const V *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (sizeof(V) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
BF_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> BF_D void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// v[r] *= w^r (r = 1..R-1), w^r = tw[r*base] (conjugated when CONJ). Radix 4
// and 8 load w, w^2 (and w^4) and form the other powers by one complex
// product each, which cuts table traffic from R-1 loads to 2 or 3.
template <int R, bool CONJ, typename V>
BF_D void apply_twiddles(V *v, const V *tw, int base) {
  if constexpr (R == 2) {
    v[1] = cmulw<CONJ>(v[1], ldtw(tw, base));
  } else if constexpr (R == 4) {
    const V w1 = ldtw(tw, base), w2 = ldtw(tw, 2 * base);
    const V w3 = cmulw<false>(w1, w2);
    v[1] = cmulw<CONJ>(v[1], w1);
    v[2] = cmulw<CONJ>(v[2], w2);
    v[3] = cmulw<CONJ>(v[3], w3);
  } else if constexpr (R == 8) {
    const V w1 = ldtw(tw, base), w2 = ldtw(tw, 2 * base), w4 = ldtw(tw, 4 * base);
    const V w3 = cmulw<false>(w1, w2);
    v[1] = cmulw<CONJ>(v[1], w1);
    v[2] = cmulw<CONJ>(v[2], w2);
    v[3] = cmulw<CONJ>(v[3], w3);
    v[4] = cmulw<CONJ>(v[4], w4);
    v[5] = cmulw<CONJ>(v[5], cmulw<false>(w4, w1));
    v[6] = cmulw<CONJ>(v[6], cmulw<false>(w4, w2));
    v[7] = cmulw<CONJ>(v[7], cmulw<false>(w4, w3));
  } else {
#pragma unroll
    for (int r = 1; r < R; ++r)
      v[r] = cmulw<CONJ>(v[r], ldtw(tw, r * base));
  }
}

// Same with a twiddle pyramid: tn points at T_n[k] = exp(-2*pi*i*k/n) and the
// tables T_{n/2}, T_{n/4} follow it (offsets n and 3n/2), so w = T_n[k],
// w^2 = T_{n/2}[k] and w^4 = T_{n/4}[k] are loads that are contiguous across
// neighbouring k.
template <int R, bool CONJ, typename V>
BF_D void apply_twiddles_pyr(V *v, const V *tn, int n, int k) {
  if constexpr (R == 2) {
    v[1] = cmulw<CONJ>(v[1], ldtw(tn, k));
  } else if constexpr (R == 4) {
    const V w1 = ldtw(tn, k), w2 = ldtw(tn, n + k);
    v[1] = cmulw<CONJ>(v[1], w1);
    v[2] = cmulw<CONJ>(v[2], w2);
    v[3] = cmulw<CONJ>(v[3], cmulw<false>(w1, w2));
  } else if constexpr (R == 8) {
    const V w1 = ldtw(tn, k), w2 = ldtw(tn, n + k), w4 = ldtw(tn, n + n / 2 + k);
    const V w3 = cmulw<false>(w1, w2);
    v[1] = cmulw<CONJ>(v[1], w1);
    v[2] = cmulw<CONJ>(v[2], w2);
    v[3] = cmulw<CONJ>(v[3], w3);
    v[4] = cmulw<CONJ>(v[4], w4);
    v[5] = cmulw<CONJ>(v[5], cmulw<false>(w4, w1));
    v[6] = cmulw<CONJ>(v[6], cmulw<false>(w4, w2));
    v[7] = cmulw<CONJ>(v[7], cmulw<false>(w4, w3));
  } else if constexpr (R == 16 || R == 32) {
    // w^(2^b) from the levels n/2^b, the other powers as products of those
    // (at most four factors for R = 32)
    V w[R];
    w[1] = ldtw(tn, k);
    w[2] = ldtw(tn, n + k);
    w[4] = ldtw(tn, n + n / 2 + k);
    w[8] = ldtw(tn, n + n / 2 + n / 4 + k);
    if constexpr (R == 32)
      w[16] = ldtw(tn, n + n / 2 + n / 4 + n / 8 + k);
    w[3] = cmulw<false>(w[1], w[2]);
#pragma unroll
    for (int r = 5; r < 8; ++r)
      w[r] = cmulw<false>(w[4], w[r - 4]);
#pragma unroll
    for (int r = 9; r < 16; ++r)
      w[r] = cmulw<false>(w[8], w[r - 8]);
    if constexpr (R == 32) {
#pragma unroll
      for (int r = 17; r < 32; ++r)
        w[r] = cmulw<false>(w[16], w[r - 16]);
    }
#pragma unroll
    for (int r = 1; r < R; ++r)
      v[r] = cmulw<CONJ>(v[r], w[r]);
  } else {
#pragma unroll
    for (int r = 1; r < R; ++r)
      v[r] = cmulw<CONJ>(v[r], ldtw(tn, (r * k) % n));
  }
}

template <typename V> BF_D V shfl_cplx(V x, int src, int width) {
  V r;
  r.x = __shfl_sync(0xffffffffu, x.x, src, width);
  r.y = __shfl_sync(0xffffffffu, x.y, src, width);
  return r;
}

// ==========================================================================
// Family S: lengths known at compile time (powers of two up to 4096).
// ==========================================================================
template <typename T, int L, int NT, int TB, bool COL, bool FWD, int KIND,
          bool STAGED = false>
struct KS {
  using V = cvec<T>;
  // radices up to the points a thread holds (32 / 16 at most)
  static constexpr SchedS<L, radix_cap(int(sizeof(V)), L, TB, NT),
                          COL ? 0 : even_row_threads(L, int(sizeof(V)), NT / TB)>
      S{};
  static constexpr int NST = S.nst;
  static constexpr int P = NT / TB; // threads per transform
  static constexpr int TSCALE = (KIND == KIND_C2C) ? 1 : 2;
  static constexpr bool WARP_SYNC = !COL && (P <= 32) && (32 % P == 0);
  static_assert(NT % TB == 0, "TB must divide NT");
  static_assert(S.rest == 1, "length not factorable");

  static constexpr int emax() {
    int e = 1;
    for (int s = 0; s < S.nst; ++s) {
      int B = L / S.rad[s];
      int K = (B + P - 1) / P;
      if (K * S.rad[s] > e)
        e = K * S.rad[s];
    }
    return e;
  }
  static constexpr int EMAX = emax();

  static constexpr bool all_full() {
    for (int s = 0; s < S.nst; ++s)
      if ((L / S.rad[s]) % P != 0)
        return false;
    return true;
  }
  // Row transforms held by P <= 32 lanes of one warp, every stage evenly
  // split: lane g owns points g + P*m, m < L/P, in the first stage's inputs
  // and the last stage's outputs. The Hermitian partner L - k of point
  // k = g + P*m then sits in lane P - g at m' = L/P - 1 - m (lane 0: its own
  // point P*(L/P - m)), so R2C/C2R pair points with warp shuffles instead of
  // a pass through shared memory.
  static constexpr bool SHUF = !COL && KIND != KIND_C2C && P <= 32 && all_full();
  // Row layouts: power-of-two lengths pad one element every 16 (8-byte
  // elements) or 8 (16-byte elements) so that both contiguous reads and the
  // stride-R writes of the Stockham stages hit every bank equally; other
  // lengths take the layout with the fewest shared-memory wavefronts on their
  // own access pattern (choose_row_pad).
  static constexpr RowPad RP = choose_row_pad(S, L, P, TB, int(sizeof(V)),
                                              KIND == KIND_R2C && !SHUF,
                                              !COL && (L & (L - 1)) != 0);
  static constexpr int PADSH = RP.sh;
  static constexpr int LP = COL ? L : RP.lp;
  static constexpr int TM = L * TSCALE; // top length of the twiddle pyramid

  static constexpr size_t smem_bytes() {
    return static_cast<size_t>(TB) * LP * sizeof(V) * (STAGED ? 2 : 1);
  }

  struct Ctx {
    int g, tb;
    bool act;
    const V *gin;
    V *gout;
    const V *tw;
    long long ist, ost;
    V *sm;
  };

  static BF_D void bar() {
    if constexpr (WARP_SYNC)
      __syncwarp();
    else
      __syncthreads();
  }
  static BF_D int sidx(const Ctx &c, int n) {
    if constexpr (COL)
      return n * TB + c.tb;
    else
      return c.tb * LP + n + (n >> PADSH);
  }

  // C2R input: Z[n] = E + i*O from X[n] and X[L-n] (real length 2L).
  // w = exp(-2*pi*i*n/(2L)).
  static BF_D V c2r_pre(const Ctx &c, int n, V w) {
    V xa = c.gin[(long long)n * c.ist];
    V xb = c.gin[(long long)(L - n) * c.ist];
    if (n == 0) {
      xa.y = T(0);
      xb.y = T(0);
    }
    V e = cadd(xa, cconj(xb));
    V o = cmulw<true>(csub(xa, cconj(xb)), w);
    return cmake(e.x - o.y, e.y + o.x);
  }

  // R2C output X[k] from za = Z[k], zb = Z[L-k], w = exp(-2*pi*i*k/(2L)):
  // X = E + w*O, E = (za + conj zb)/2, O = -i (za - conj zb)/2.
  static BF_D V r2c_from_pair(V za, V zb, V w) {
    const V b = cconj(zb);
    const V e = cmake(T(0.5) * (za.x + b.x), T(0.5) * (za.y + b.y));
    const V d = csub(za, b);
    const V o = cmake(T(0.5) * d.y, T(-0.5) * d.x);
    return cadd(e, cmulw<false>(o, w));
  }

  // C2R input Z[n] from xa = X[n], xb = X[L-n], w = exp(-2*pi*i*n/(2L)):
  // Z = E + i*O, E = xa + conj xb, O = (xa - conj xb) * conj(w).
  static BF_D V c2r_from_pair(V xa, V xb, V w) {
    const V e = cadd(xa, cconj(xb));
    const V o = cmulw<true>(csub(xa, cconj(xb)), w);
    return cmake(e.x - o.y, e.y + o.x);
  }

  // R2C output k in [0, L] from Z held in shared memory (natural order).
  // w = exp(-2*pi*i*k/(2L)).
  static BF_D V r2c_post(const Ctx &c, int k, V w) {
    V a = c.sm[sidx(c, k == L ? 0 : k)];
    V b = cconj(c.sm[sidx(c, k == 0 ? 0 : L - k)]);
    V e = cmake(T(0.5) * (a.x + b.x), T(0.5) * (a.y + b.y));
    V d = csub(a, b);
    V o = cmake(T(0.5) * d.y, T(-0.5) * d.x); // -i*(a-b)/2
    return cadd(e, cmulw<false>(o, w));
  }

  template <int s> static BF_D void run(Ctx &c, V (&v)[EMAX]) {
    constexpr int R = S.rad[s];
    constexpr int Ns = S.ns[s];
    constexpr int B = L / R;
    constexpr int K = (B + P - 1) / P;
    constexpr bool FULL = (B % P) == 0;
    if constexpr (s > 0) {
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
        if (FULL || j < B) {
          const int k = j % Ns;
          if constexpr ((L & (L - 1)) == 0) // pyramid: level Ns*R at offset 2TM - 2Ns*R
            apply_twiddles_pyr<R, !FWD>(&v[i * R], c.tw + (2 * TM - 2 * Ns * R), Ns * R, k);
          else // flat table of TM entries: w^(r k) at r * k * TM / (Ns R)
            apply_twiddles<R, !FWD>(&v[i * R], c.tw, k * (TM / (Ns * R)));
        }
      }
    }
#pragma unroll
    for (int i = 0; i < K; ++i)
      dft<R, FWD>(&v[i * R]);

    if constexpr (s == NST - 1) {
      if constexpr (KIND == KIND_R2C && SHUF) {
        // lane g holds Z[g + P*m] in v[(m % BP)*R + m / BP]
        constexpr int NM = L / P;
        constexpr int BP = B / P;
        const int src = (P - c.g) & (P - 1);
#pragma unroll
        for (int m = 0; m < NM; ++m) {
          const int mp = NM - 1 - m;
          V zb = shfl_cplx(v[(mp % BP) * R + mp / BP], src, P);
          if (c.g == 0) {
            const int m2 = (NM - m) % NM;
            zb = v[(m2 % BP) * R + m2 / BP];
          }
          const V za = v[(m % BP) * R + m / BP];
          const V w = ldtw(c.tw, c.g + P * m); // coalesced table read
          if (c.act)
            c.gout[(long long)(c.g + P * m) * c.ost] = r2c_from_pair(za, zb, w);
        }
        if (c.act && c.g == 0) // X[L] = Re Z[0] - Im Z[0]
          c.gout[(long long)L * c.ost] = cmake(v[0].x - v[0].y, T(0));
      } else if constexpr (KIND == KIND_R2C) {
        if constexpr (s > 0)
          bar();
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const int j = c.g + P * i;
          if (FULL || j < B) {
#pragma unroll
            for (int r = 0; r < R; ++r)
              c.sm[sidx(c, j + r * B)] = v[i * R + r];
          }
        }
        bar();
        // exp(-2*pi*i*(g + P*i)/(2L)) = tw[g] * tw[P*i]; tw[P*i] is the
        // same for every thread (a broadcast load).
        constexpr int KO = (L + 1 + P - 1) / P;
        const V wg = ldtw(c.tw, c.g);
#pragma unroll
        for (int i = 0; i < KO; ++i) {
          const int k = c.g + P * i;
          if (c.act && k <= L)
            c.gout[(long long)k * c.ost] =
                r2c_post(c, k, i == 0 ? wg : cmulw<false>(wg, ldtw(c.tw, P * i)));
        }
      } else {
        if (c.act) {
#pragma unroll
          for (int i = 0; i < K; ++i) {
            const int j = c.g + P * i;
            if (FULL || j < B) {
#pragma unroll
              for (int r = 0; r < R; ++r)
                c.gout[(long long)(j + r * B) * c.ost] = v[i * R + r];
            }
          }
        }
      }
    } else {
      if constexpr (s > 0 || STAGED)
        bar();
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
        if (FULL || j < B) {
          const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
          for (int r = 0; r < R; ++r)
            c.sm[sidx(c, base + r * Ns)] = v[i * R + r];
        }
      }
      bar();
      constexpr int R2 = S.rad[s + 1];
      constexpr int B2 = L / R2;
      constexpr int K2 = (B2 + P - 1) / P;
      constexpr bool FULL2 = (B2 % P) == 0;
#pragma unroll
      for (int i = 0; i < K2; ++i) {
        const int j = c.g + P * i;
        if (FULL2 || j < B2) {
#pragma unroll
          for (int r = 0; r < R2; ++r)
            v[i * R2 + r] = c.sm[sidx(c, j + r * B2)];
        }
      }
      run<s + 1>(c, v);
    }
  }

  // Tile `tile` (TB transforms) of the pass.
  static BF_D void entry(const PassArgs &a, V *sm, long long tile) {
    Ctx c;
    const int tid = threadIdx.x;
    c.g = COL ? (tid / TB) : (tid % P);
    c.tb = COL ? (tid % TB) : (tid / P);
    const long long b = tile * TB + c.tb;
    c.act = b < a.total;
    long long ioff = 0, ooff = 0;
    if (c.act) {
      long long sl, w;
      slab_of(a, b, sl, w);
      ioff = sl * a.islab + w * a.idist;
      ooff = sl * a.oslab + w * a.odist;
    }
    c.gin = reinterpret_cast<const V *>(a.in) + ioff;
    c.gout = reinterpret_cast<V *>(a.out) + ooff;
    c.tw = reinterpret_cast<const V *>(a.tw);
    // R2C/C2R rows are contiguous (unit stride, checked by the planner): a
    // constant stride lets every load and store fold its offset.
    c.ist = KIND == KIND_C2C ? a.istride : 1;
    c.ost = KIND == KIND_C2C ? a.ostride : 1;
    c.sm = sm;

    V v[EMAX];
    constexpr int R = S.rad[0];
    constexpr int B = L / R;
    constexpr int K = (B + P - 1) / P;
    constexpr bool FULL = (B % P) == 0;
    if constexpr (KIND == KIND_C2R && SHUF) {
      // lane g loads X[g + P*m] (coalesced) and lane 0 also X[L]; the
      // partner X[L - n] comes from lane P - g by shuffle.
      constexpr int NM = L / P;
      constexpr int BP = B / P;
      V x[NM];
#pragma unroll
      for (int m = 0; m < NM; ++m)
        x[m] = c.act ? c.gin[(long long)(c.g + P * m) * c.ist] : czero<V>();
      const V xl = (c.act && c.g == 0) ? c.gin[(long long)L * c.ist] : czero<V>();
      const int src = (P - c.g) & (P - 1);
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        V xb = shfl_cplx(x[NM - 1 - m], src, P);
        V xa = x[m];
        if (c.g == 0) {
          xb = m == 0 ? xl : x[NM - m];
          if (m == 0) { // Im of DC and Nyquist are ignored
            xa.y = T(0);
            xb.y = T(0);
          }
        }
        const V w = ldtw(c.tw, c.g + P * m); // coalesced table read
        v[(m % BP) * R + m / BP] = c2r_from_pair(xa, xb, w);
      }
      run<0>(c, v);
      return;
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int j = c.g + P * i;
      const bool ok = c.act && (FULL || j < B);
      V wj;
      if constexpr (KIND == KIND_C2R)
        wj = ldtw(c.tw, j < B ? j : 0);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int n = j + r * B;
        if constexpr (KIND == KIND_C2R) // tw[j + r*B] = tw[j] * tw[r*B]
          v[i * R + r] =
              ok ? c2r_pre(c, n, r == 0 ? wj : cmulw<false>(wj, ldtw(c.tw, r * B)))
                 : czero<V>();
        else
          v[i * R + r] = ok ? c.gin[(long long)n * c.ist] : czero<V>();
      }
    }
    run<0>(c, v);
  }

  // ---- persistent column pass with register prefetch ----------------------
  // Each CTA walks tiles blockIdx.x, +gridDim.x, ...; the points of the next
  // tile are loaded into a second register set before the current tile is
  // transformed, so global loads stay in flight through the compute phase.
  // Shared memory holds one exchange buffer per register set.
  static BF_D void set_tile(Ctx &c, const PassArgs &a, long long tile) {
    const long long b = tile * TB + c.tb;
    c.act = b < a.total;
    long long ioff = 0, ooff = 0;
    if (c.act) {
      long long sl, w;
      slab_of(a, b, sl, w);
      ioff = sl * a.islab + w * a.idist;
      ooff = sl * a.oslab + w * a.odist;
    }
    c.gin = reinterpret_cast<const V *>(a.in) + ioff;
    c.gout = reinterpret_cast<V *>(a.out) + ooff;
  }
  static BF_D void load_first(const Ctx &c, V (&v)[EMAX]) {
    constexpr int R = S.rad[0];
    constexpr int B = L / R;
    constexpr int K = (B + P - 1) / P;
    constexpr bool FULL = (B % P) == 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int j = c.g + P * i;
      const bool ok = c.act && (FULL || j < B);
#pragma unroll
      for (int r = 0; r < R; ++r)
        v[i * R + r] = ok ? c.gin[(long long)(j + r * B) * c.ist] : czero<V>();
    }
  }
  static BF_D void entry_pipelined(const PassArgs &a, V *smem) {
    static_assert(COL && KIND == KIND_C2C, "pipelined path is for column C2C");
    const long long ntiles = (a.total + TB - 1) / TB;
    const long long G = gridDim.x;
    long long t = blockIdx.x;
    if (t >= ntiles)
      return;
    Ctx ca, cb;
    const int tid = threadIdx.x;
    ca.g = cb.g = tid / TB;
    ca.tb = cb.tb = tid % TB;
    ca.tw = cb.tw = reinterpret_cast<const V *>(a.tw);
    ca.ist = cb.ist = a.istride;
    ca.ost = cb.ost = a.ostride;
    ca.sm = smem;
    cb.sm = smem + static_cast<size_t>(L) * TB;
    V va[EMAX], vb[EMAX];
    set_tile(ca, a, t);
    load_first(ca, va);
    for (; t < ntiles; t += 2 * G) {
      set_tile(cb, a, t + G); // inactive (no loads) past the last tile
      load_first(cb, vb);
      run<0>(ca, va);
      if (t + G >= ntiles)
        break;
      set_tile(ca, a, t + 2 * G);
      load_first(ca, va);
      run<0>(cb, vb);
    }
  }

  // ---- persistent column pass with cp.async double buffering -------------
  // CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...; while tile t is
  // transformed in one shared buffer, the points of the next tile stream into
  // the other, so loads stay in flight through the compute phases. Each tile
  // holds TB adjacent transforms, L points each, as [point][transform].
  static BF_D void prefetch(const PassArgs &a, V *buf, long long tile) {
    static_assert(NT % TB == 0, "whole rows per pass");
    const int tb = threadIdx.x % TB;
    const int n0 = threadIdx.x / TB;
    const long long b = tile * TB + tb;
    if (b >= a.total)
      return;
    long long sl, w;
    slab_of(a, b, sl, w);
    const V *g = reinterpret_cast<const V *>(a.in) + sl * a.islab + w * a.idist;
    constexpr int ROWS = NT / TB;
#pragma unroll 8
    for (int n = n0; n < L; n += ROWS)
      cp_async_elem(buf + n * TB + tb, g + static_cast<long long>(n) * a.istride);
  }

  static BF_D void entry_staged(const PassArgs &a, V *smem) {
    static_assert(COL && KIND == KIND_C2C && STAGED, "staged path is for column C2C");
    const long long ntiles = (a.total + TB - 1) / TB;
    long long tile = blockIdx.x;
    if (tile >= ntiles)
      return;
    V *const buf0 = smem;
    V *const buf1 = smem + static_cast<size_t>(L) * TB;
    prefetch(a, buf0, tile);
    cp_async_commit();
    Ctx c;
    const int tid = threadIdx.x;
    c.g = tid / TB;
    c.tb = tid % TB;
    c.tw = reinterpret_cast<const V *>(a.tw);
    c.ist = a.istride;
    c.ost = a.ostride;
    c.gin = nullptr;
    for (int it = 0;; ++it) {
      const long long next = tile + gridDim.x;
      if (next < ntiles)
        prefetch(a, (it & 1) ? buf0 : buf1, next);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
      c.sm = (it & 1) ? buf1 : buf0;
      const long long b = tile * TB + c.tb;
      c.act = b < a.total;
      long long ooff = 0;
      if (c.act) {
        long long sl, w;
        slab_of(a, b, sl, w);
        ooff = sl * a.oslab + w * a.odist;
      }
      c.gout = reinterpret_cast<V *>(a.out) + ooff;
      V v[EMAX];
      constexpr int R = S.rad[0];
      constexpr int B = L / R;
      constexpr int K = (B + P - 1) / P;
      constexpr bool FULL = (B % P) == 0;
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
        if (FULL || j < B) {
#pragma unroll
          for (int r = 0; r < R; ++r)
            v[i * R + r] = c.sm[sidx(c, j + r * B)];
        }
      }
      run<0>(c, v);
      __syncthreads(); // this buffer is refilled two tiles from now
      tile = next;
      if (tile >= ntiles)
        break;
    }
  }
};

// 256-thread column kernels keep two CTAs per SM (at most 128 registers):
// left alone, the compiler hoists the twiddle loads of later stages and
// drops to one CTA per SM, which halves the loads in flight.
#ifndef B2_COL_MIN_BLOCKS
#define B2_COL_MIN_BLOCKS 2
#endif
#ifndef B2_ROW_MIN_BLOCKS
#define B2_ROW_MIN_BLOCKS 2
#endif
// 512-thread FP32 column tiles with at most 16 points per thread fit two
// CTAs per SM (64 registers; FP64 points need twice the registers).
// 256-thread row tiles with at most 8 points per thread (R2C/C2R of 512 reals,
// C2C of 256 points) fit four CTAs per SM (64 registers).
template <int ES, int NT, int TB, int L, bool COL> constexpr int static_min_blocks() {
  return NT == 256 ? (COL ? B2_COL_MIN_BLOCKS
                          : ((TB * L) / NT <= 8 && ES == 8    ? 4
                             : (TB * L) / NT <= 16 && ES == 8 ? 3
                                                              : B2_ROW_MIN_BLOCKS))
                   : ((ES == 8 && COL && NT == 512 && (TB * L) / NT <= 16) ? 2 : 1);
}
template <typename T, int L, int NT, int TB, bool COL, bool FWD, int KIND>
__global__ void __launch_bounds__(NT, (static_min_blocks<int(sizeof(T) * 2), NT, TB, L, COL>()))
    fft_static_kernel(const PassArgs a) {
  using K = KS<T, L, NT, TB, COL, FWD, KIND>;
  extern __shared__ __align__(16) unsigned char smraw[];
  K::entry(a, reinterpret_cast<typename K::V *>(smraw), blockIdx.x);
}

// Grouped specialised pass: the same length and layout for many independent
// passes (items, e.g. the same stage of many separate grids), each with its
// own pointers, batch and strides. CTA blockIdx.x runs global tile
// blockIdx.x: tile_map[blockIdx.x] = (item, tile within the item), built on
// the host, so a CTA finds its work with one load.
template <typename T, int L, int NT, int TB, bool COL, bool FWD, int KIND>
__global__ void __launch_bounds__(NT, (static_min_blocks<int(sizeof(T) * 2), NT, TB, L, COL>()))
    fft_static_group_kernel(const PassArgs *__restrict__ items,
                            const int2 *__restrict__ tile_map) {
  using K = KS<T, L, NT, TB, COL, FWD, KIND>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int2 m = tile_map[blockIdx.x];
  const PassArgs a = items[m.x];
  K::entry(a, reinterpret_cast<typename K::V *>(smraw), m.y);
}

template <typename T, int L, int NT, int TB, bool FWD>
__global__ void __launch_bounds__(NT, 2)
    fft_static_pipelined_kernel(const PassArgs a) {
  using K = KS<T, L, NT, TB, true, FWD, KIND_C2C>;
  extern __shared__ __align__(16) unsigned char smraw[];
  K::entry_pipelined(a, reinterpret_cast<typename K::V *>(smraw));
}

template <typename T, int L, int NT, int TB, bool FWD>
__global__ void __launch_bounds__(NT)
    fft_static_staged_kernel(const PassArgs a) {
  using K = KS<T, L, NT, TB, true, FWD, KIND_C2C, true>;
  extern __shared__ __align__(16) unsigned char smraw[];
  K::entry_staged(a, reinterpret_cast<typename K::V *>(smraw));
}

// ==========================================================================
// Family G: runtime length and radix schedule (any length whose prime
// factors are 2, 3, 5, 7 or another prime <= kGenMaxPrime).
// ==========================================================================
template <bool COL> BF_D int gidx(int tb, int n, int TB, int L) {
  return COL ? n * TB + tb : tb * L + n;
}

// Generic stage butterflies. `ld(n)` returns point n of the stage input and
// `st(n, v)` stores point n of its output: shared memory between stages,
// global memory in the first stage's loads and the last stage's stores.
template <int R, bool FWD, typename V, class Ld, class St>
BF_D void gen_butterfly(const GenArgs &a, Ld &&ld, St &&st, const V *tw, int j, int k, int Bq,
                        int Ns, int texp) {
  V v[R];
#pragma unroll
  for (int r = 0; r < R; ++r)
    v[r] = ld(j + r * Bq);
  if (Ns > 1)
    apply_twiddles<R, !FWD>(v, tw, k * texp * a.tscale);
  dft<R, FWD>(v);
  const int base = (j - k) * R + k; // (j/Ns)*Ns*R + k
#pragma unroll
  for (int r = 0; r < R; ++r)
    st(base + r * Ns, v[r]);
}

// Prime radix p by direct summation; DFT constants come from the table:
// exp(-2*pi*i*r*m/p) = tw[((r*m) mod p) * (L/p) * tscale].
template <bool FWD, typename V, class Ld, class St>
BF_D void gen_butterfly_prime(const GenArgs &a, Ld &&ld, St &&st, const V *tw, int p, int j,
                              int k, int Bq, int Ns, int texp) {
  V x[kGenMaxPrime];
  for (int r = 0; r < p; ++r) {
    V t = ld(j + r * Bq);
    if (r > 0 && Ns > 1)
      t = cmulw<!FWD>(t, ldtw(tw, r * k * texp * a.tscale));
    x[r] = t;
  }
  const int step = (a.L / p) * a.tscale;
  const int base = (j - k) * p + k;
  for (int m = 0; m < p; ++m) {
    V acc = x[0];
    int e = 0;
    for (int r = 1; r < p; ++r) {
      e += m;
      if (e >= p)
        e -= p;
      acc = cadd(acc, cmulw<!FWD>(x[r], ldtw(tw, e * step)));
    }
    st(base + m * Ns, acc);
  }
}

template <bool FWD, typename V, class Ld, class St>
BF_D void gen_radix(const GenArgs &a, int R, Ld &&ld, St &&st, const V *tw, int j, int k, int Bq,
                    int Ns, int texp) {
  switch (R) {
  case 2: gen_butterfly<2, FWD>(a, ld, st, tw, j, k, Bq, Ns, texp); break;
  case 3: gen_butterfly<3, FWD>(a, ld, st, tw, j, k, Bq, Ns, texp); break;
  case 4: gen_butterfly<4, FWD>(a, ld, st, tw, j, k, Bq, Ns, texp); break;
  case 5: gen_butterfly<5, FWD>(a, ld, st, tw, j, k, Bq, Ns, texp); break;
  case 8: gen_butterfly<8, FWD>(a, ld, st, tw, j, k, Bq, Ns, texp); break;
  default: gen_butterfly_prime<FWD>(a, ld, st, tw, R, j, k, Bq, Ns, texp); break;
  }
}

// One tile (a.TB transforms) of a generic pass, run by a whole CTA of
// kGenThreads threads with 2*TB*L elements of dynamic shared memory. The
// first stage reads its points from global memory and (except for R2C, whose
// Hermitian post-process pairs outputs k and L-k) the last stage writes
// global memory, so a tile crosses shared memory once per stage boundary.
template <typename T, bool COL, int KIND, bool FWD>
BF_D void gen_tile(const GenArgs &a, long long tile, unsigned char *smraw) {
  using V = cvec<T>;
  V *A = reinterpret_cast<V *>(smraw);
  V *Bm = A + static_cast<size_t>(a.TB) * a.L;
  const V *tw = reinterpret_cast<const V *>(a.p.tw);
  const int tid = threadIdx.x;
  const int TB = a.TB, L = a.L;
  const long long tile0 = tile * TB;

  // Offsets of the tile's transforms, computed once per tile (one 64-bit
  // division each) instead of once per element. -1: beyond the batch.
  __shared__ long long s_io[kGenMaxTB], s_oo[kGenMaxTB];
  if (tid < TB) {
    const long long b = tile0 + tid;
    long long io = -1, oo = -1;
    if (b < a.p.total) {
      const long long sl = b / a.p.batch;
      const long long w = b - sl * a.p.batch;
      io = sl * a.p.islab + w * a.p.idist;
      oo = sl * a.p.oslab + w * a.p.odist;
    }
    s_io[tid] = io;
    s_oo[tid] = oo;
  }
  __syncthreads();

  // Point n of transform tb of the pass input (zero beyond the batch).
  auto gload = [&](int tb, int n) -> V {
    const long long io = s_io[tb];
    V val = czero<V>();
    if (io < 0)
      return val;
    const long long is = a.p.istride;
    if constexpr (KIND == KIND_C2C) {
      val = reinterpret_cast<const V *>(a.p.in)[io + n * is];
    } else if constexpr (KIND == KIND_R2C) {
      const T *x = reinterpret_cast<const T *>(a.p.in) + io;
      if (a.odd)
        val = cmake(x[n * is], T(0));
      else
        val = cmake(x[(2LL * n) * is], x[(2LL * n + 1) * is]);
    } else { // C2R
      const V *X = reinterpret_cast<const V *>(a.p.in) + io;
      if (a.odd) {
        const int nh = a.nreal / 2;
        if (n <= nh) {
          val = X[n * is];
          if (n == 0)
            val.y = T(0);
        } else {
          val = cconj(X[(long long)(a.nreal - n) * is]);
        }
      } else {
        V xa = X[n * is];
        V xb = X[(long long)(L - n) * is];
        if (n == 0) {
          xa.y = T(0);
          xb.y = T(0);
        }
        V ev = cadd(xa, cconj(xb));
        V ov = cmulw<true>(csub(xa, cconj(xb)), ldtw(tw, n));
        val = cmake(ev.x - ov.y, ev.y + ov.x);
      }
    }
    return val;
  };
  // Point k of transform tb of a C2C or C2R pass output.
  auto gstore = [&](int tb, int k, V z) {
    const long long oo = s_oo[tb];
    if (oo < 0)
      return;
    const long long os = a.p.ostride;
    if constexpr (KIND == KIND_C2C) {
      reinterpret_cast<V *>(a.p.out)[oo + k * os] = z;
    } else if constexpr (KIND == KIND_C2R) {
      T *x = reinterpret_cast<T *>(a.p.out) + oo;
      if (a.odd) {
        x[k * os] = z.x;
      } else {
        x[(2LL * k) * os] = z.x;
        x[(2LL * k + 1) * os] = z.y;
      }
    }
  };

  const bool direct_in = a.nst > 0;
  const bool direct_out = a.nst > 0 && KIND != KIND_R2C;

  // ---- load (only for a length without stages) -----------------------------
  if (!direct_in) {
    for (int e = tid; e < TB * L; e += kGenThreads) {
      int tb, n;
      if (COL) {
        tb = e & (TB - 1);
        n = e >> a.logTB;
      } else {
        tb = static_cast<int>(fdiv(static_cast<uint32_t>(e), a.Ldiv));
        n = e - tb * L;
      }
      A[gidx<COL>(tb, n, TB, L)] = gload(tb, n);
    }
    __syncthreads();
  }

  // ---- stages ---------------------------------------------------------------
  for (int s = 0; s < a.nst; ++s) {
    const int R = a.rad[s];
    const int Ns = a.nsv[s];
    const int Bq = L / R;
    const int texp = L / (Ns * R);
    const int cnt = TB * Bq;
    const bool first = s == 0;
    const bool last = s == a.nst - 1 && direct_out;
    for (int q = tid; q < cnt; q += kGenThreads) {
      int tb, j;
      if (COL) {
        tb = q & (TB - 1);
        j = q >> a.logTB;
      } else {
        tb = static_cast<int>(fdiv(static_cast<uint32_t>(q), a.bq[s]));
        j = q - tb * Bq;
      }
      const int k = j - static_cast<int>(fdiv(static_cast<uint32_t>(j), a.ns[s])) * Ns;
      auto ld_s = [&](int n) { return A[gidx<COL>(tb, n, TB, L)]; };
      auto ld_g = [&](int n) { return gload(tb, n); };
      auto st_s = [&](int n, V v) { Bm[gidx<COL>(tb, n, TB, L)] = v; };
      auto st_g = [&](int n, V v) { gstore(tb, n, v); };
      if (first && last)
        gen_radix<FWD>(a, R, ld_g, st_g, tw, j, k, Bq, Ns, texp);
      else if (first)
        gen_radix<FWD>(a, R, ld_g, st_s, tw, j, k, Bq, Ns, texp);
      else if (last)
        gen_radix<FWD>(a, R, ld_s, st_g, tw, j, k, Bq, Ns, texp);
      else
        gen_radix<FWD>(a, R, ld_s, st_s, tw, j, k, Bq, Ns, texp);
    }
    if (last)
      return; // the caller synchronises before the next tile reuses shared memory
    __syncthreads();
    V *t = A;
    A = Bm;
    Bm = t;
  }

  // ---- store (R2C, and lengths without stages) ------------------------------
  const int lout = a.lout;
  for (int e = tid; e < TB * lout; e += kGenThreads) {
    int tb, k;
    if (COL) {
      tb = e & (TB - 1);
      k = e >> a.logTB;
    } else {
      tb = static_cast<int>(fdiv(static_cast<uint32_t>(e), a.Loutdiv));
      k = e - tb * lout;
    }
    const long long oo = s_oo[tb];
    if (oo < 0)
      continue;
    const long long os = a.p.ostride;
    if constexpr (KIND == KIND_R2C) {
      V *X = reinterpret_cast<V *>(a.p.out) + oo;
      if (a.odd) {
        X[k * os] = A[gidx<COL>(tb, k, TB, L)];
      } else {
        V za = A[gidx<COL>(tb, k == L ? 0 : k, TB, L)];
        V zb = cconj(A[gidx<COL>(tb, k == 0 ? 0 : L - k, TB, L)]);
        V ev = cmake(T(0.5) * (za.x + zb.x), T(0.5) * (za.y + zb.y));
        V d = csub(za, zb);
        V ov = cmake(T(0.5) * d.y, T(-0.5) * d.x);
        X[k * os] = cadd(ev, cmulw<false>(ov, ldtw(tw, k)));
      }
    } else {
      gstore(tb, k, A[gidx<COL>(tb, k, TB, L)]);
    }
  }
}

template <typename T, bool COL, int KIND, bool FWD>
__global__ void __launch_bounds__(kGenThreads) fft_generic_kernel(const GenArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  gen_tile<T, COL, KIND, FWD>(a, blockIdx.x, smraw);
}

// Persistent grouped pass: CTAs take tiles from a device work queue (one
// atomic counter) until all tiles of all items are done. Item i covers tiles
// [tile_start[i], tile_start[i+1]); items are passes of independent
// transforms (for example the same stage of many separate grids), each with
// its own length, layout, pointers and twiddle table.
template <typename T, bool COL, int KIND, bool FWD>
__global__ void __launch_bounds__(kGenThreads)
    fft_generic_group_kernel(const GenArgs *__restrict__ items,
                             const long long *__restrict__ tile_start, int nitems,
                             unsigned long long *queue) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ long long task_s[2];
  __shared__ int item_s[2];
  const long long ntasks = tile_start[nitems];
  // Map a claimed tile number to its item (binary search on tile_start).
  auto resolve = [&](long long t, int slot) {
    int lo = 0, hi = nitems - 1;
    if (t < ntasks) {
      while (lo < hi) { // last item whose first tile is <= t
        const int mid = (lo + hi + 1) >> 1;
        if (tile_start[mid] <= t)
          lo = mid;
        else
          hi = mid - 1;
      }
    }
    task_s[slot] = t;
    item_s[slot] = lo;
  };
  if (threadIdx.x == 0)
    resolve(static_cast<long long>(atomicAdd(queue, 1ull)), 0);
  __syncthreads();
  for (int it = 0;; ++it) {
    const int cur = it & 1;
    const long long t = task_s[cur];
    const int i = item_s[cur];
    if (t >= ntasks)
      return;
    // The next claim is issued now and resolved after this tile, so the
    // atomic's round trip overlaps the tile's work.
    unsigned long long next = 0;
    if (threadIdx.x == 0)
      next = atomicAdd(queue, 1ull);
    gen_tile<T, COL, KIND, FWD>(items[i], t - tile_start[i], smraw);
    if (threadIdx.x == 0)
      resolve(static_cast<long long>(next), cur ^ 1);
    __syncthreads(); // shared memory and the next task are ready
  }
}

} // namespace b200fft
