// Column tiles with two neighbouring transforms per thread (FP32 C2C,
// power-of-two lengths): tile variant kVariantPair.
//
// The column tile of Family S (KS, COL) gives each thread the points of one
// transform. Here each thread holds the same points of two neighbouring
// transforms (2p, 2p+1) of its tile, so
//   * every shared-memory exchange moves 16 bytes per access (the tile's
//     layout [point][transform] keeps the two side by side): half the
//     shared-memory instructions;
//   * the stage twiddles, which depend only on the point index, are loaded
//     and formed once for both transforms;
//   * where the two transforms are adjacent in memory at a 16-byte aligned
//     address on every point row (VEC: unit transform distance, even point
//     stride, even slab stride, batch even so no pair spans two slabs, both
//     bases 16-byte aligned), global loads and stores move 16 bytes too.
// Elsewhere (odd point strides, such as the middle axis of a padded R2C
// grid, 257 complex) global accesses stay 8 bytes wide (VEC = false) and a
// thread's pair is transforms p and p + TB/2 of the tile, so that each load
// or store instruction of a warp still covers contiguous runs of a point row;
// such pairs may span two slabs.
// The Stockham stage structure is that of KS (fft_device.cuh).
#pragma once

#include "fft_device.cuh"

namespace b200fft {

// w[r] = w^r (r = 1..R-1) of w = T_n[k] from a twiddle pyramid (T_n, then
// T_{n/2}, T_{n/4}, ...), conjugated when CONJ.
template <int R, bool CONJ>
BF_D void pyr_powers(float2 (&w)[R], const float2 *tn, int n, int k) {
  w[1] = ldtw(tn, k);
  if constexpr (R >= 4)
    w[2] = ldtw(tn, n + k);
  if constexpr (R >= 8)
    w[4] = ldtw(tn, n + n / 2 + k);
  if constexpr (R >= 16)
    w[8] = ldtw(tn, n + n / 2 + n / 4 + k);
  if constexpr (R >= 4)
    w[3] = cmulw<false>(w[1], w[2]);
  if constexpr (R >= 8) {
#pragma unroll
    for (int r = 5; r < 8; ++r)
      w[r] = cmulw<false>(w[4], w[r - 4]);
  }
  if constexpr (R >= 16) {
#pragma unroll
    for (int r = 9; r < 16; ++r)
      w[r] = cmulw<false>(w[8], w[r - 8]);
  }
  if constexpr (CONJ) {
#pragma unroll
    for (int r = 1; r < R; ++r)
      w[r].y = -w[r].y;
  }
}

template <int L, int NT, int TB, bool FWD, bool VEC> struct KP {
  using V = float2;
  static constexpr int TP = TB / 2;   // transform pairs per tile
  static constexpr int P = NT / TP;   // threads per pair column
  static constexpr int E = L / P;     // points per transform per thread
  static_assert(TB % 2 == 0 && NT % TP == 0 && L % P == 0, "pair tile shape");
  static constexpr SchedS<L, (E >= 16 ? 16 : 8), 0> S{};
  static constexpr int NST = S.nst;
  static constexpr int TM = L;        // top length of the twiddle pyramid
  static_assert(S.rest == 1, "length not factorable");

  static constexpr int emax() {
    int e = 1;
    for (int s = 0; s < S.nst; ++s) {
      const int K = (L / S.rad[s]) / P;
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
  static_assert(all_full(), "every stage fills all threads");

  static constexpr size_t smem_bytes() { return static_cast<size_t>(L) * TB * sizeof(V); }

  struct Ctx {
    int g, tp;
    bool act0, act1;
    const V *in0, *in1; // the pair's first points (in1 unused when VEC)
    V *out0, *out1;
    const V *tw;
    long long ist, ost;
    float4 *sm;
  };

  static BF_D float4 pack(V a, V b) { return make_float4(a.x, a.y, b.x, b.y); }

  template <int s> static BF_D void run(Ctx &c, V (&va)[EMAX], V (&vb)[EMAX]) {
    constexpr int R = S.rad[s];
    constexpr int Ns = S.ns[s];
    constexpr int B = L / R;
    constexpr int K = B / P;
    if constexpr (s > 0) {
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
        V w[R];
        pyr_powers<R, !FWD>(w, c.tw + (2 * TM - 2 * Ns * R), Ns * R, j % Ns);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          va[i * R + r] = cmulw<false>(va[i * R + r], w[r]);
          vb[i * R + r] = cmulw<false>(vb[i * R + r], w[r]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      dft<R, FWD>(&va[i * R]);
      dft<R, FWD>(&vb[i * R]);
    }
    if constexpr (s == NST - 1) {
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const long long o = static_cast<long long>(j + r * B) * c.ost;
          if constexpr (VEC) {
            if (c.act0)
              *reinterpret_cast<float4 *>(c.out0 + o) = pack(va[i * R + r], vb[i * R + r]);
          } else {
            if (c.act0)
              c.out0[o] = va[i * R + r];
            if (c.act1)
              c.out1[o] = vb[i * R + r];
          }
        }
      }
    } else {
      if constexpr (s > 0)
        __syncthreads();
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int j = c.g + P * i;
        const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
        for (int r = 0; r < R; ++r)
          c.sm[(base + r * Ns) * TP + c.tp] = pack(va[i * R + r], vb[i * R + r]);
      }
      __syncthreads();
      constexpr int R2 = S.rad[s + 1];
      constexpr int B2 = L / R2;
      constexpr int K2 = B2 / P;
#pragma unroll
      for (int i = 0; i < K2; ++i) {
        const int j = c.g + P * i;
#pragma unroll
        for (int r = 0; r < R2; ++r) {
          const float4 q = c.sm[(j + r * B2) * TP + c.tp];
          va[i * R2 + r] = make_float2(q.x, q.y);
          vb[i * R2 + r] = make_float2(q.z, q.w);
        }
      }
      run<s + 1>(c, va, vb);
    }
  }

  static BF_D void entry(const PassArgs &a, float4 *sm, long long tile) {
    Ctx c;
    const int tid = threadIdx.x;
    c.g = tid / TP;
    c.tp = tid % TP;
    // the pair: transforms (2p, 2p+1) with 16-byte accesses, else (p, p+TP)
    const long long b0 = tile * TB + (VEC ? 2 * c.tp : c.tp);
    const long long b1 = VEC ? b0 + 1 : b0 + TP;
    c.act0 = b0 < a.total;
    c.act1 = b1 < a.total;
    long long i0 = 0, o0 = 0, i1 = 0, o1 = 0;
    if (c.act0) {
      long long sl, w;
      slab_of(a, b0, sl, w);
      i0 = sl * a.islab + w * a.idist;
      o0 = sl * a.oslab + w * a.odist;
    }
    if (!VEC && c.act1) {
      long long sl, w;
      slab_of(a, b1, sl, w);
      i1 = sl * a.islab + w * a.idist;
      o1 = sl * a.oslab + w * a.odist;
    }
    const V *in = reinterpret_cast<const V *>(a.in);
    V *out = reinterpret_cast<V *>(a.out);
    c.in0 = in + i0;
    c.in1 = in + i1;
    c.out0 = out + o0;
    c.out1 = out + o1;
    c.tw = reinterpret_cast<const V *>(a.tw);
    c.ist = a.istride;
    c.ost = a.ostride;
    c.sm = sm;

    V va[EMAX], vb[EMAX];
    constexpr int R = S.rad[0];
    constexpr int B = L / R;
    constexpr int K = B / P;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int j = c.g + P * i;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const long long o = static_cast<long long>(j + r * B) * c.ist;
        if constexpr (VEC) {
          float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
          if (c.act0)
            q = *reinterpret_cast<const float4 *>(c.in0 + o);
          va[i * R + r] = make_float2(q.x, q.y);
          vb[i * R + r] = make_float2(q.z, q.w);
        } else {
          va[i * R + r] = c.act0 ? c.in0[o] : czero<V>();
          vb[i * R + r] = c.act1 ? c.in1[o] : czero<V>();
        }
      }
    }
    run<0>(c, va, vb);
  }
};

template <int L, int NT, int TB, bool FWD, bool VEC>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 2) fft_colpair_kernel(const PassArgs a) {
  using K = KP<L, NT, TB, FWD, VEC>;
  extern __shared__ __align__(16) unsigned char smraw[];
  K::entry(a, reinterpret_cast<float4 *>(smraw), blockIdx.x);
}

} // namespace b200fft
