// Split-precision tensor-core transforms ("split-TC"): FP32 C2C of length
// 256, 512 and 1024 whose radix-16 DFT blocks run on the tensor cores as
// dense complex matrix products with FP16 operands split into hi + lo parts
// and FP32 accumulation (mma.sync m16n8k16).
//
// 256 = 16 x 16 four-step. In one m16n8k16 product the A operand is the
// DFT-16 matrix (rows: outputs; K: inputs), the B operand holds 8 vectors of
// 16 points, and the accumulator holds their 16-point DFTs:
//   B fragment of lane (g, t) = (lane >> 2, lane & 3): vector g, input
//     slots {2t, 2t+1, 2t+8, 2t+9};
//   accumulator: outputs {g, g+8} of vectors {2t, 2t+1}.
// Real and imaginary parts take separate k-tiles and m-tiles:
//   Re = C xr + S xi,  Im = -S xr + C xi,  C = cos(2 pi k n / 16),
//   S = +-sin(2 pi k n / 16) (sign by direction).
// Step 1 transforms over n1 (X index 16 n1 + n2), the W256^(k1 n2) twiddle
// is applied in FP32, and step 2 transforms over n2, giving X[k1 + 16 k2].
//
// Split precision: operands are scaled by a power of two (a block exponent)
// so that every FP16 value stays inside the FP16 range, and each operand v is
// split v = hi + lo, hi = fp16(v), lo = fp16(v - hi), about 22 of FP32's 24
// bits. Each product is formed as A_lo B_hi + A_hi B_lo + A_hi B_hi with FP32
// accumulation; A_lo B_lo lies below FP32 rounding. The tensor cores truncate
// their FP32 sums, so the two large products end separate accumulators (one
// truncation each) and are added in FP32 with rounding to nearest.
// Constants come from the FP64-generated twiddle table of the plain kernels
// (pyramid levels 16, 256 and L).
//
// Lengths 512 and 1024 take one decimation-in-frequency radix-2 / radix-4
// step in FP32 first, y_p[n] = W_L^(n p) sum_q W_R0^(p q) x[n + 256 q], then
// a 256-point four-step on each y_p gives X[R0 k + p].
//
// Row transforms (points contiguous): one warp per transform, in registers.
// Lane (g, t) takes points n = 16 (2t+h+8r) + g + 8j (+ 256 q): the B
// fragments of step 1 with vectors n2 = g + 8j; its step-1 accumulators
// (k1 in {g, g+8}, n2 in {2t, 2t+1} + 8j) are register for register the B
// fragments of step 2 (vectors k1, slots n2), so the corner turn of the
// four-step moves no data; the outputs k = 2t + h + 8jp + 16 (g + 8hh) leave
// as contiguous 16-byte stores. One block exponent per 256-point block.
//
// Column transforms (points strided, neighbouring transforms adjacent): a
// CTA takes 16 neighbouring transforms, so every point row is one 128-byte
// segment. The 16 vectors of a product are the 16 columns (n-tile j holds
// columns 2g + j), which lane (g, t) loads as one 16-byte pair. Step 1 runs
// per n2 from global memory and writes the twiddled FP32 results to shared
// memory; after one barrier step 2 runs per (block, k1) from shared memory
// and writes global memory directly. Block exponents are per column and per
// step (the quad of lanes holding a column agrees on it).
#include <cuda_fp16.h>

#include <climits>
#include <stdint.h>

#include "fft_device.cuh"
#include "launch.hpp"

namespace b200fft {
namespace {

BF_D uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t *>(&h); }

// Split two FP32 values into packed FP16 hi and lo parts (a in the low half).
BF_D void split2(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 f = __half22float2(h);
  hi = h2u(h);
  lo = h2u(__floats2half2_rn(a - f.x, b - f.y));
}

// d += A * B, A 16x16 row-major FP16, B 16x8 column-major FP16, d FP32.
BF_D void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The DFT-16 matrices C, S and -S as hi/lo A fragments. Register i of lane
// (g, t) holds rows g (+8 if i & 1) and columns 2t, 2t+1 (+8 if i & 2).
struct TcConst {
  uint32_t ch[4], cl[4], sh[4], sl[4], nh[4], nl[4];
};

template <bool FWD> BF_D void tc_setup(TcConst &K, const float2 *tw16, int g, int t) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = g + ((i & 1) ? 8 : 0);
    const int col = 2 * t + ((i & 2) ? 8 : 0);
    float c[2], s[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float2 w = __ldg(tw16 + ((row * (col + h)) & 15));
      c[h] = w.x;
      s[h] = FWD ? -w.y : w.y; // forward: sin(theta) = -Im exp(-i theta)
    }
    split2(c[0], c[1], K.ch[i], K.cl[i]);
    split2(s[0], s[1], K.sh[i], K.sl[i]);
    split2(-s[0], -s[1], K.nh[i], K.nl[i]);
  }
}

// Complex DFT-16 of one n-tile: dr = C br + S bi, di = -S br + C bi.
BF_D void cmma(const TcConst &K, float (&dr)[4], float (&di)[4], const uint32_t (&brh)[2],
               const uint32_t (&brl)[2], const uint32_t (&bih)[2], const uint32_t (&bil)[2]) {
  float r1[4] = {0.f, 0.f, 0.f, 0.f}, r2[4] = {0.f, 0.f, 0.f, 0.f};
  float i1[4] = {0.f, 0.f, 0.f, 0.f}, i2[4] = {0.f, 0.f, 0.f, 0.f};
  mma16816(r2, K.cl, brh[0], brh[1]);
  mma16816(i2, K.nl, brh[0], brh[1]);
  mma16816(r2, K.ch, brl[0], brl[1]);
  mma16816(i2, K.nh, brl[0], brl[1]);
  mma16816(r2, K.sl, bih[0], bih[1]);
  mma16816(i2, K.cl, bih[0], bih[1]);
  mma16816(r2, K.sh, bil[0], bil[1]);
  mma16816(i2, K.ch, bil[0], bil[1]);
  mma16816(r1, K.ch, brh[0], brh[1]);
  mma16816(i1, K.nh, brh[0], brh[1]);
  mma16816(r2, K.sh, bih[0], bih[1]);
  mma16816(i2, K.ch, bih[0], bih[1]);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dr[i] = r1[i] + r2[i];
    di[i] = i1[i] + i2[i];
  }
}

// Scale 2^(lim - e) for a block whose largest magnitude m lies in
// [2^e, 2^(e+1)), clamped so that the scale and its inverse are normal.
BF_D void block_scale(float m, int lim, float &s, float &inv) {
  int sb = 127 + lim + 127 - ((__float_as_int(m) >> 23) & 0xff);
  sb = sb < 1 ? 1 : (sb > 253 ? 253 : sb);
  s = __int_as_float(sb << 23);
  inv = __int_as_float((254 - sb) << 23);
}

BF_D float amax(float2 v) { return fmaxf(fabsf(v.x), fabsf(v.y)); }

template <bool FWD> BF_D float2 tw_at(const float2 *tw, int m) {
  float2 w = __ldg(tw + m);
  if (!FWD)
    w.y = -w.y;
  return w;
}

// Radix-R0 decimation-in-frequency step over v[q] = x[n + 256 q]; on return
// v[p] = W_L^(n p) sum_q W_R0^(p q) v[q].
template <int R0, bool FWD>
BF_D void dif_step(float2 (&v)[R0], const float2 *twL, int n) {
  if constexpr (R0 == 2)
    dft2<FWD>(v[0], v[1]);
  else if constexpr (R0 == 4)
    dft4<FWD>(v[0], v[1], v[2], v[3]);
#pragma unroll
  for (int p = 1; p < R0; ++p)
    v[p] = cmulw<!FWD>(v[p], __ldg(twL + n * p));
}

// ---------------------------------------------------------------------------
// Row transforms: one warp, one 256-point block in registers.
// In:  x[j*4 + r*2 + h] = point 16 (2t + h + 8r) + g + 8j.
// Out: x[jp*4 + hh*2 + h] = point (2t + h + 8jp) + 16 (g + 8hh).
template <bool FWD>
BF_D void row_w256(const TcConst &K, const float2 *tw256, float2 (&x)[8], int g, int t) {
  float m = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    m = fmaxf(m, amax(x[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // |step-1 input| < 2^11, so |step-2 input| <= 16 * 2^11 = 2^15 < 65504
  float s, inv;
  block_scale(m, 10, s, inv);
  float2 y[8];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    uint32_t brh[2], brl[2], bih[2], bil[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const float2 a = x[j * 4 + r * 2], b = x[j * 4 + r * 2 + 1];
      split2(a.x * s, b.x * s, brh[r], brl[r]);
      split2(a.y * s, b.y * s, bih[r], bil[r]);
    }
    float dr[4], di[4];
    cmma(K, dr, di, brh, brl, bih, bil);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int k1 = g + ((c & 2) ? 8 : 0);
      const int n2 = 2 * t + (c & 1) + 8 * j;
      y[j * 4 + c] = cmulw<false>(make_float2(dr[c], di[c]), tw_at<FWD>(tw256, (k1 * n2) & 255));
    }
  }
#pragma unroll
  for (int jp = 0; jp < 2; ++jp) {
    uint32_t brh[2], brl[2], bih[2], bil[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const float2 a = y[r * 4 + 2 * jp], b = y[r * 4 + 2 * jp + 1];
      split2(a.x, b.x, brh[r], brl[r]);
      split2(a.y, b.y, bih[r], bil[r]);
    }
    float dr[4], di[4];
    cmma(K, dr, di, brh, brl, bih, bil);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      x[jp * 4 + c] = make_float2(dr[c] * inv, di[c] * inv);
  }
}

// 512- and 1024-point rows hold 16 and 32 points per lane: three 4-warp CTAs
// per SM leave them room.
template <int L> constexpr int row_min_blocks() { return L >= 512 ? 3 : 4; }
constexpr int kRowWarps = 4;

// Each warp walks transforms b, b + (all warps), ...: it loads the points of
// its fragments straight from global memory (every load instruction covers
// full 32-byte sectors), transforms them in registers and stores 16-byte
// runs of the output.
template <int L, bool FWD>
__global__ void __launch_bounds__(kRowWarps * 32, row_min_blocks<L>())
    fft_tc_row_kernel(PassArgs a) {
  constexpr int R0 = L / 256;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const float2 *tw = static_cast<const float2 *>(a.tw);
  const float2 *tw256 = tw + (2 * L - 512); // pyramid level n at offset 2L - 2n
  TcConst K;
  tc_setup<FWD>(K, tw + (2 * L - 32), g, t);
  const long long nwarp = static_cast<long long>(gridDim.x) * kRowWarps;
#pragma unroll 1
  for (long long b = static_cast<long long>(blockIdx.x) * kRowWarps + (threadIdx.x >> 5);
       b < a.total; b += nwarp) {
    long long sl, w;
    slab_of(a, b, sl, w);
    const float2 *in = static_cast<const float2 *>(a.in) + sl * a.islab + w * a.idist;
    float2 *out = static_cast<float2 *>(a.out) + sl * a.oslab + w * a.odist;
    const long long is = a.istride, os = a.ostride;
    float2 x[R0][8];
#pragma unroll
    for (int q = 0; q < R0; ++q)
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int j = i >> 2, r = (i >> 1) & 1, h = i & 1;
        const int n = 256 * q + 16 * (2 * t + h + 8 * r) + g + 8 * j;
        x[q][i] = in[n * is];
      }
    if constexpr (R0 > 1) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int j = i >> 2, r = (i >> 1) & 1, h = i & 1;
        const int n = 16 * (2 * t + h + 8 * r) + g + 8 * j;
        float2 v[R0];
#pragma unroll
        for (int q = 0; q < R0; ++q)
          v[q] = x[q][i];
        dif_step<R0, FWD>(v, tw, n);
#pragma unroll
        for (int p = 0; p < R0; ++p)
          x[p][i] = v[p];
      }
    }
#pragma unroll
    for (int p = 0; p < R0; ++p)
      row_w256<FWD>(K, tw256, x[p], g, t);
    // X[R0 k + p] with k = 2t + h + 8jp + 16 (g + 8hh): for each (jp, hh) the
    // lane holds 2 R0 consecutive outputs starting at R0 (2t + 8jp + 16 (g + 8hh)).
    const bool vec = os == 1 && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
#pragma unroll
    for (int jp = 0; jp < 2; ++jp)
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int k0 = 2 * t + 8 * jp + 16 * (g + 8 * hh);
        if (vec) {
          float4 *o4 = reinterpret_cast<float4 *>(out + R0 * k0);
#pragma unroll
          for (int v = 0; v < R0; ++v) { // outputs R0 k0 + 2v, + 2v + 1
            const int e0 = 2 * v, e1 = 2 * v + 1;
            const float2 u0 = x[e0 % R0][jp * 4 + hh * 2 + e0 / R0];
            const float2 u1 = x[e1 % R0][jp * 4 + hh * 2 + e1 / R0];
            o4[v] = make_float4(u0.x, u0.y, u1.x, u1.y);
          }
        } else {
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int p = 0; p < R0; ++p)
              out[(R0 * (k0 + h) + p) * os] = x[p][jp * 4 + hh * 2 + h];
        }
      }
  }
}

// ---------------------------------------------------------------------------
// Column transforms.
template <int L> struct ColCfg {
  static constexpr int R0 = L / 256;
  static constexpr int NT = L == 1024 ? 512 : 256;
  static constexpr int NW = NT / 32;
  static constexpr size_t smem = static_cast<size_t>(L) * 16 * sizeof(float2);
};

// Shared-memory slot of Y[p][k1][n2][column c]: 16-byte column pairs are
// swizzled by n2 and k1 so that the step-1 writes and the step-2 reads are
// free of bank conflicts.
BF_D int yidx(int p, int k1, int n2, int c) {
  const int chunk = (c >> 1) ^ (((n2 >> 1) & 3) << 1) ^ (k1 & 1);
  return (((p * 16 + k1) * 16 + n2) * 16) + chunk * 2 + (c & 1);
}

// Per-column block exponents of an n-tile pair: lanes 4n..4n+3 hold the
// slots of columns 2n (a) and 2n + 1 (b).
BF_D void col_scales(float ma, float mb, int lim, float &sa, float &sb, float &ia, float &ib) {
  ma = fmaxf(ma, __shfl_xor_sync(0xffffffffu, ma, 1));
  ma = fmaxf(ma, __shfl_xor_sync(0xffffffffu, ma, 2));
  mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, 1));
  mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, 2));
  block_scale(ma, lim, sa, ia);
  block_scale(mb, lim, sb, ib);
}

// DFT-16 of the 16 columns of one slot set. va/vb[r*2 + h]: slot 2t + h + 8r
// of columns 2g (a) and 2g + 1 (b). Result: d{re,im}[j][c] = output
// g + 8 (c >> 1) of column 2 (2t + (c & 1)) + j, descaled.
BF_D void col_dft16(const TcConst &K, const float2 (&va)[4], const float2 (&vb)[4], int t,
                    float (&dre)[2][4], float (&dim)[2][4]) {
  float ma = 0.f, mb = 0.f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    ma = fmaxf(ma, amax(va[i]));
    mb = fmaxf(mb, amax(vb[i]));
  }
  float sa, sb, ia, ib;
  // outputs stay FP32, so inputs may use the whole FP16 range: max*s < 2^15
  col_scales(ma, mb, 14, sa, sb, ia, ib);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float2(&v)[4] = j ? vb : va;
    const float s = j ? sb : sa;
    uint32_t brh[2], brl[2], bih[2], bil[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      split2(v[r * 2].x * s, v[r * 2 + 1].x * s, brh[r], brl[r]);
      split2(v[r * 2].y * s, v[r * 2 + 1].y * s, bih[r], bil[r]);
    }
    cmma(K, dre[j], dim[j], brh, brl, bih, bil);
    // inverse scales of columns 2(2t) + j and 2(2t + 1) + j
    const float inv_own = j ? ib : ia;
    const float i0 = __shfl_sync(0xffffffffu, inv_own, 4 * (2 * t));
    const float i1 = __shfl_sync(0xffffffffu, inv_own, 4 * (2 * t + 1));
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float iv = (c & 1) ? i1 : i0;
      dre[j][c] *= iv;
      dim[j][c] *= iv;
    }
  }
}

template <int L, bool FWD>
__global__ void __launch_bounds__(ColCfg<L>::NT, ColCfg<L>::NT == 512 ? 1 : 2)
    fft_tc_col_kernel(PassArgs a) {
  using Cf = ColCfg<L>;
  constexpr int R0 = Cf::R0, NW = Cf::NW;
  extern __shared__ __align__(16) unsigned char tc_smraw[];
  float2 *Y = reinterpret_cast<float2 *>(tc_smraw);
  __shared__ long long s_in[16], s_out[16];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const float2 *tw = static_cast<const float2 *>(a.tw);
  const float2 *tw256 = tw + (2 * L - 512);
  TcConst K;
  tc_setup<FWD>(K, tw + (2 * L - 32), g, t);
  const float2 *gin = static_cast<const float2 *>(a.in);
  float2 *gout = static_cast<float2 *>(a.out);
  const long long is = a.istride, os = a.ostride;
  const long long ntiles = (a.total + 15) / 16;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (tid < 16) {
      const long long b = tile * 16 + tid;
      long long io = -1, oo = -1;
      if (b < a.total) {
        long long sl, w;
        slab_of(a, b, sl, w);
        io = sl * a.islab + w * a.idist;
        oo = sl * a.oslab + w * a.odist;
      }
      s_in[tid] = io;
      s_out[tid] = oo;
    }
    __syncthreads();
    // ---- step 1: per n2, DFT-16 over n1 for every block p and column
    {
      const long long pa = s_in[2 * g], pb = s_in[2 * g + 1];
      // 16-byte pair loads when the two columns are adjacent and every row
      // of the pair stays 16-byte aligned (even stride)
      const bool vin = pa >= 0 && pb == pa + 1 && (is & 1) == 0 &&
                       ((reinterpret_cast<uintptr_t>(gin + pa) & 15) == 0);
#pragma unroll 1
      for (int n2 = warp; n2 < 16; n2 += NW) {
        float2 xa[R0][4], xb[R0][4];
#pragma unroll
        for (int q = 0; q < R0; ++q)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = i >> 1, h = i & 1;
            const long long e = 256 * q + 16 * (2 * t + h + 8 * r) + n2;
            if (vin) {
              const float4 v = *reinterpret_cast<const float4 *>(gin + pa + e * is);
              xa[q][i] = make_float2(v.x, v.y);
              xb[q][i] = make_float2(v.z, v.w);
            } else {
              xa[q][i] = pa >= 0 ? gin[pa + e * is] : make_float2(0.f, 0.f);
              xb[q][i] = pb >= 0 ? gin[pb + e * is] : make_float2(0.f, 0.f);
            }
          }
        if constexpr (R0 > 1) {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = i >> 1, h = i & 1;
            const int n = 16 * (2 * t + h + 8 * r) + n2;
            float2 va[R0], vb[R0];
#pragma unroll
            for (int q = 0; q < R0; ++q) {
              va[q] = xa[q][i];
              vb[q] = xb[q][i];
            }
            dif_step<R0, FWD>(va, tw, n);
            dif_step<R0, FWD>(vb, tw, n);
#pragma unroll
            for (int p = 0; p < R0; ++p) {
              xa[p][i] = va[p];
              xb[p][i] = vb[p];
            }
          }
        }
        const float2 w0 = tw_at<FWD>(tw256, (g * n2) & 255);
        const float2 w1 = tw_at<FWD>(tw256, ((g + 8) * n2) & 255);
#pragma unroll
        for (int p = 0; p < R0; ++p) {
          float dre[2][4], dim[2][4];
          col_dft16(K, xa[p], xb[p], t, dre, dim);
          // rows k1 = g (c = 0, 1) and g + 8 (c = 2, 3); columns 4t + 2 (c & 1) + j
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            const int k1 = g + 8 * hh;
            const float2 w = hh ? w1 : w0;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
              const int c = hh * 2 + cc;
              const float2 u0 = cmulw<false>(make_float2(dre[0][c], dim[0][c]), w);
              const float2 u1 = cmulw<false>(make_float2(dre[1][c], dim[1][c]), w);
              *reinterpret_cast<float4 *>(Y + yidx(p, k1, n2, 4 * t + 2 * cc)) =
                  make_float4(u0.x, u0.y, u1.x, u1.y);
            }
          }
        }
      }
    }
    __syncthreads();
    // ---- step 2: per (p, k1), DFT-16 over n2; X[R0 (k1 + 16 k2) + p]
    {
      long long po[4];
      bool vout[2];
#pragma unroll
      for (int v = 0; v < 4; ++v)
        po[v] = s_out[4 * t + v];
#pragma unroll
      for (int cc = 0; cc < 2; ++cc)
        vout[cc] = po[2 * cc] >= 0 && po[2 * cc + 1] == po[2 * cc] + 1 && (os & 1) == 0 &&
                   ((reinterpret_cast<uintptr_t>(gout + po[2 * cc]) & 15) == 0);
#pragma unroll 1
      for (int pk = warp; pk < R0 * 16; pk += NW) {
        const int p = pk >> 4, k1 = pk & 15;
        float2 va[4], vb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = i >> 1, h = i & 1;
          const float4 v =
              *reinterpret_cast<const float4 *>(Y + yidx(p, k1, 2 * t + h + 8 * r, 2 * g));
          va[i] = make_float2(v.x, v.y);
          vb[i] = make_float2(v.z, v.w);
        }
        float dre[2][4], dim[2][4];
        col_dft16(K, va, vb, t, dre, dim);
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const long long row = R0 * (k1 + 16 * (g + 8 * hh)) + p;
#pragma unroll
          for (int cc = 0; cc < 2; ++cc) {
            const int c = hh * 2 + cc;
            const float2 u0 = make_float2(dre[0][c], dim[0][c]);
            const float2 u1 = make_float2(dre[1][c], dim[1][c]);
            const long long o0 = po[2 * cc], o1 = po[2 * cc + 1];
            if (vout[cc]) {
              *reinterpret_cast<float4 *>(gout + o0 + row * os) =
                  make_float4(u0.x, u0.y, u1.x, u1.y);
            } else {
              if (o0 >= 0)
                gout[o0 + row * os] = u0;
              if (o1 >= 0)
                gout[o1 + row * os] = u1;
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// Per-device launch set-up: opt into large shared memory and size the
// persistent grid from the occupancy of the kernel.
template <typename Kern>
cudaError_t prepare(Kern kern, int nt, size_t smem, int *slots_out, int *mask, int *per_sm) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 31)
    return cudaErrorInvalidDevice;
  if (!(*mask & (1 << dev))) {
    if (smem > 48 * 1024) {
      const cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess)
        return e;
    }
    int nb = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, nt, smem);
    if (e != cudaSuccess)
      return e;
    per_sm[dev] = nb > 0 ? nb : 1;
    *mask |= (1 << dev);
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  *slots_out = per_sm[dev] * sms;
  return cudaSuccess;
}

template <int L, bool FWD> cudaError_t launch_row(const PassArgs &a, cudaStream_t st) {
  auto kern = fft_tc_row_kernel<L, FWD>;
  static int mask = 0, per_sm[32] = {0};
  int slots = 0;
  const cudaError_t e = prepare(kern, kRowWarps * 32, 0, &slots, &mask, per_sm);
  if (e != cudaSuccess)
    return e;
  const long long blocks = (a.total + kRowWarps - 1) / kRowWarps;
  if (blocks <= 0)
    return cudaSuccess;
  const long long grid = blocks < slots ? blocks : slots;
  kern<<<static_cast<unsigned>(grid), kRowWarps * 32, 0, st>>>(a);
  return cudaGetLastError();
}

template <int L, bool FWD> cudaError_t launch_col(const PassArgs &a, cudaStream_t st) {
  using Cf = ColCfg<L>;
  auto kern = fft_tc_col_kernel<L, FWD>;
  static int mask = 0, per_sm[32] = {0};
  int slots = 0;
  const cudaError_t e = prepare(kern, Cf::NT, Cf::smem, &slots, &mask, per_sm);
  if (e != cudaSuccess)
    return e;
  const long long ntiles = (a.total + 15) / 16;
  if (ntiles <= 0)
    return cudaSuccess;
  const long long grid = ntiles < slots ? ntiles : slots;
  kern<<<static_cast<unsigned>(grid), Cf::NT, Cf::smem, st>>>(a);
  return cudaGetLastError();
}

template <int L>
cudaError_t launch_len(bool col, bool fwd, const PassArgs &a, cudaStream_t st) {
  if (col)
    return fwd ? launch_col<L, true>(a, st) : launch_col<L, false>(a, st);
  return fwd ? launch_row<L, true>(a, st) : launch_row<L, false>(a, st);
}

} // namespace

cudaError_t launch_tc_c2c_f32(int L, bool col, bool fwd, const PassArgs &a, cudaStream_t st) {
  switch (L) {
  case 256: return launch_len<256>(col, fwd, a, st);
  case 512: return launch_len<512>(col, fwd, a, st);
  case 1024: return launch_len<1024>(col, fwd, a, st);
  default: return cudaErrorInvalidValue;
  }
}

} // namespace b200fft
