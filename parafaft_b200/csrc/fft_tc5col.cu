// Split-precision tensor-core 512-point columns on the fifth-generation
// tensor cores (tcgen05): FP32 C2C, columns (points strided, neighbouring
// transforms adjacent), the split-TC form of the middle and first axes of a
// 512^3 grid.
//
// 512 = 16 x 32 four-step, n = 32 n1 + n2, k = k1 + 16 k2:
//   step 1: Y[n2][k1]  = sum_n1 x[32 n1 + n2] W16^(n1 k1)        (DFT-16, K = 16)
//   twiddle: Y'[n2][k1] = Y[n2][k1] W512^(n2 k1)                  (FP32)
//   step 2: X[k1 + 16 k2] = sum_n2 Y'[n2][k1] W32^(n2 k2)        (DFT-32, K = 32)
// Each DFT block is a complex matrix product with FP16 hi + lo operands
// (A_lo B_hi + A_hi B_lo + A_hi B_hi), FP32 accumulation, the two large
// products in separate accumulators, as in the 256-point row kernel
// (fft_tc5.cu). The complex product is one real product per output half: the
// real and imaginary parts of A are two K-blocks, B holds (c, -s) / (s, c)
// rows, N = 16 real + 16 imaginary outputs. Every product is
//   D[128 x 32] = A[128 x 16] * B[16 x 32]   (kind::f16, M = 128, N = 32).
// A tile is 16 neighbouring transforms (128-byte row segments), 512 threads:
//   step 1: thread (t, n2) = tid (tid = 16 n2 + t) owns row 32 (warp % 4) + lane
//           of M-block warp / 4 (rows (t, n2), four M-blocks), loads its 16
//           points x_t[32 n1 + n2] (one warp reads two 128-byte row segments
//           per load), scales them by its own block exponent and stores its
//           K-major row;
//   step 2: rows (t, k1) (two M-blocks, row 16 t + k1), K = n2 in two K-blocks,
//           written by the step-1 threads as MN-major operands (16-byte
//           stores); one block exponent per transform (its 32 rows);
//   output: each thread reads one (row, output half) of the products and
//           stages X through shared memory (row pitch 17, no bank conflicts),
//           then the CTA writes whole 128-byte row segments.
// Operand layouts are the canonical no-swizzle layouts of tc5_common.cuh.
// TMEM: 256 columns (step 2 reuses step 1's after they are read), so two
// CTAs run per SM; shared memory (88 KiB) allows no third.
//
// Every wait on the product barrier is bounded by the clock: past the limit
// the CTA records a fault in a device word (read back by the host at
// b200fft_sync as B200FFT_ERR_DEVICE_STATUS), frees its tensor memory and
// returns.
#include <cuda_fp16.h>

#include <atomic>
#include <cstdlib>
#include <stdint.h>

#include "fft_device.cuh"
#include "launch.hpp"
#include "tc5_common.cuh"

namespace b200fft {
namespace {

using namespace tc5;

__device__ unsigned int g_tc5col_fault = 0;

constexpr int kCThreads = 512;
constexpr int kCTB = 16;             // transforms per tile
constexpr uint32_t kCCols = 256;     // TMEM columns per CTA
constexpr int kReg = 4096;           // one 128 x 16 FP16 operand region
constexpr int kRegB = 1024;          // one 32 x 16 FP16 operand region
constexpr int kPitch = 17;           // output staging row pitch (float2)
constexpr int kAreaBytes = 512 * kPitch * 8;      // A operands, then output staging
constexpr int kB1Off = kAreaBytes;                // DFT-16: 4 regions
constexpr int kB2Off = kB1Off + 4 * kRegB;        // DFT-32: (half, K-block) x 4 regions
constexpr int kSmemBytes = kB2Off + 16 * kRegB;   // 90112 bytes
static_assert(4 * 4 * kReg <= kAreaBytes, "step-1 operands fit the area");

// The six products of one K-block into accumulators a (hi re * hi) and b
// (the rest); `first` starts both accumulators (K-block 0).
BF_D void issue6(uint32_t d, const unsigned char *A, const unsigned char *B, bool a_mn,
                 bool first) {
  const uint32_t id = idesc_f16(a_mn, 128, 32);
  auto ad = [&](int r) { return umma_desc(smem_u32(A + r * kReg), 128u, 256u); };
  auto bd = [&](int r) { return umma_desc(smem_u32(B + r * kRegB), 128u, 256u); };
  const uint32_t acc_a = d, acc_b = d + 32;
  const uint32_t f = first ? 0u : 1u;
  umma(acc_b, ad(2), bd(0), id, f); // lo re * hi
  umma(acc_b, ad(0), bd(2), id, 1); // hi re * lo
  umma(acc_b, ad(3), bd(1), id, 1); // lo im * hi
  umma(acc_b, ad(1), bd(3), id, 1); // hi im * lo
  umma(acc_b, ad(1), bd(1), id, 1); // hi im * hi
  umma(acc_a, ad(0), bd(0), id, f); // hi re * hi
}

// Store one complex DFT matrix entry, split into hi and lo, at row n, column
// k of the 4-region B block at `B` (regions: 0 hi re-part, 1 hi im-part, 2 lo
// re-part, 3 lo im-part). Row n < 16 gives real outputs, n >= 16 imaginary.
BF_D void put_b(unsigned char *B, int n, int k, float c, float s) {
#pragma unroll
  for (int kb = 0; kb < 2; ++kb) {
    const float val = kb == 0 ? (n < 16 ? c : -s) : (n < 16 ? s : c);
    const __half hi = __float2half_rn(val);
    const __half lo = __float2half_rn(val - __half2float(hi));
    const int off = kmaj(n, k);
    *reinterpret_cast<__half *>(B + (0 + kb) * kRegB + off) = hi;
    *reinterpret_cast<__half *>(B + (2 + kb) * kRegB + off) = lo;
  }
}

// Split 8 complex values (a 16-byte chunk of each region) and store them.
BF_D void put_a8(unsigned char *A, int off, const float2 *x, float s) {
  uint32_t hr[4], lr[4], hi[4], li[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 p0 = x[2 * q], p1 = x[2 * q + 1];
    split2(p0.x * s, p1.x * s, hr[q], lr[q]);
    split2(p0.y * s, p1.y * s, hi[q], li[q]);
  }
  *reinterpret_cast<uint4 *>(A + 0 * kReg + off) = make_uint4(hr[0], hr[1], hr[2], hr[3]);
  *reinterpret_cast<uint4 *>(A + 1 * kReg + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  *reinterpret_cast<uint4 *>(A + 2 * kReg + off) = make_uint4(lr[0], lr[1], lr[2], lr[3]);
  *reinterpret_cast<uint4 *>(A + 3 * kReg + off) = make_uint4(li[0], li[1], li[2], li[3]);
}

// stall != 0 (a host-side test switch) issues no products and waits on a
// barrier phase that nothing completes, so the bounded wait runs out and the
// fault path is exercised without any GPU fault.
template <bool FWD>
__global__ void __launch_bounds__(kCThreads, 2) fft_tc5_col512_kernel(PassArgs a, int stall) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *const area = smem;
  unsigned char *const B1 = smem + kB1Off;
  unsigned char *const B2 = smem + kB2Off;
  float2 *const stage = reinterpret_cast<float2 *>(smem);
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_s;
  __shared__ int abort_s;
  __shared__ int mx[kCTB]; // per-transform step-2 maxima (float bits, >= 0)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = tid & 15, n2 = tid >> 4;     // step-1 row (t, n2)
  const int mb1 = warp >> 2;                 // its M-block
  const int m1 = 32 * (warp & 3) + lane;     // its row in the M-block
  const float2 *tw = static_cast<const float2 *>(a.tw);
  const uint32_t mb = smem_u32(&mbar);

  // ---- set-up: TMEM, barrier, the DFT-16 and DFT-32 operands ---------------
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_s)),
                 "r"(kCCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_s = 0;
  }
  // B1: DFT-16 (level 16 of the 512 pyramid at 2*512 - 32), N = k1 (re, im)
  for (int i = tid; i < 32 * 16; i += kCThreads) {
    const int k = i & 15, n = i >> 4;
    const float2 w = __ldg(tw + (2 * 512 - 32) + (((n & 15) * k) & 15));
    put_b(B1, n, k, w.x, FWD ? -w.y : w.y);
  }
  // B2: DFT-32 (level 32 at 2*512 - 64); block (h, kb): outputs k2 = 16 h +
  // (n & 15), inputs n2 = 16 kb + k
  for (int i = tid; i < 4 * 32 * 16; i += kCThreads) {
    const int k = i & 15, n = (i >> 4) & 31, hk = i >> 9; // hk = 2 h + kb
    const int k2 = 16 * (hk >> 1) + (n & 15), nn2 = 16 * (hk & 1) + k;
    const float2 w = __ldg(tw + (2 * 512 - 64) + ((k2 * nn2) & 31));
    put_b(B2 + hk * 4 * kRegB, n, k, w.x, FWD ? -w.y : w.y);
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_s;
  const uint32_t tquad = tmem + (static_cast<uint32_t>(32 * (warp & 3)) << 16);
  uint32_t phase = 0;

  const long long ntiles = (a.total + kCTB - 1) / kCTB;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long b = tile * kCTB + t;
    const bool act = b < a.total;
    long long io = 0, oo = 0;
    if (act) {
      long long sl, w;
      slab_of(a, b, sl, w);
      io = sl * a.islab + w * a.idist;
      oo = sl * a.oslab + w * a.odist;
    }
    const float2 *in = static_cast<const float2 *>(a.in) + io;
    float2 *out = static_cast<float2 *>(a.out) + oo;
    if (tid < kCTB)
      mx[tid] = 0;

    // ---- step 1 operand: row (t, n2), K = n1 -------------------------------
    float2 x[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1)
      x[n1] = act ? in[static_cast<long long>(32 * n1 + n2) * a.istride] : make_float2(0.f, 0.f);
    float m = 0.f;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1)
      m = fmaxf(m, fmaxf(fabsf(x[n1].x), fabsf(x[n1].y)));
    float s1, inv1;
    block_scale(m, 14, s1, inv1);
    unsigned char *const A1 = area + mb1 * 4 * kReg;
    put_a8(A1, kmaj(m1, 0), x, s1);
    put_a8(A1, kmaj(m1, 8), x + 8, s1);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      if (!stall) {
#pragma unroll
        for (int blk = 0; blk < 4; ++blk)
          issue6(tmem + 64 * blk, area + blk * 4 * kReg, B1, false, true);
        umma_commit(mb);
      }
      if (!mbar_wait(mb, phase))
        abort_s = 1;
    }
    phase ^= 1;
    fence_after();
    __syncthreads();
    if (abort_s)
      break;

    // ---- twiddle; step 2 operand: rows (t, k1), K = n2 (MN-major) ----------
    float2 y[16];
    float m2 = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float re[8], im[8];
      tmem_outputs8(tquad + 64 * mb1, h, re, im);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k1 = 8 * h + i;
        float2 w = __ldg(tw + ((n2 * k1) & 511)); // level 512 at offset 0
        if (!FWD)
          w.y = -w.y;
        y[k1] = cmulw<false>(make_float2(re[i] * inv1, im[i] * inv1), w);
        m2 = fmaxf(m2, fmaxf(fabsf(y[k1].x), fabsf(y[k1].y)));
      }
    }
    // one block exponent per transform: its 32 step-1 rows (lanes t, t + 16
    // of every warp)
    m2 = fmaxf(m2, __shfl_xor_sync(0xffffffffu, m2, 16));
    if (lane < 16)
      atomicMax(&mx[t], __float_as_int(m2));
    fence_before(); // the step-1 accumulators are read before step 2 reuses them
    __syncthreads();
    float s2, inv2;
    block_scale(__int_as_float(mx[t]), 14, s2, inv2);
    {
      // row 16 t + k1 of M-block t / 8 (lane 16 (t % 8) + k1), column n2 of
      // K-block n2 / 16
      unsigned char *const A2 = area + ((t >> 3) * 2 + (n2 >> 4)) * 4 * kReg;
      const int mrow = 16 * (t & 7);
      put_a8(A2, mnmaj(mrow, n2 & 15), y, s2);
      put_a8(A2, mnmaj(mrow + 8, n2 & 15), y + 8, s2);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
#pragma unroll
      for (int blk = 0; blk < 2; ++blk)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int kb = 0; kb < 2; ++kb)
            issue6(tmem + 128 * blk + 64 * h, area + (blk * 2 + kb) * 4 * kReg,
                   B2 + (2 * h + kb) * 4 * kRegB, true, kb == 0);
      umma_commit(mb);
      if (!mbar_wait(mb, phase))
        abort_s = 1;
    }
    phase ^= 1;
    fence_after();
    __syncthreads();
    if (abort_s)
      break;

    // ---- outputs: warp w reads (row block, half) w / 4 of its lane quarter,
    //      stages X[t][k1 + 16 k2] at [k1 + 16 k2][t] ------------------------
    {
      const int c = warp >> 2, blk = c >> 1, h = c & 1;
      const int q = 128 * blk + 32 * (warp & 3) + lane; // step-2 row 16 t + k1
      const int to = q >> 4, k1 = q & 15;
      float s2o, inv2o;
      block_scale(__int_as_float(mx[to]), 14, s2o, inv2o);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        float re[8], im[8];
        tmem_outputs8(tquad + 128 * blk + 64 * h, j, re, im);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int k2 = 16 * h + 8 * j + i;
          stage[(k1 + 16 * k2) * kPitch + to] = make_float2(re[i] * inv2o, im[i] * inv2o);
        }
      }
    }
    fence_before(); // TMEM reads done before the next tile's products
    __syncthreads();
    if (act) {
#pragma unroll 4
      for (int i = 0; i < 16; ++i) {
        const int p = n2 + 32 * i;
        out[static_cast<long long>(p) * a.ostride] = stage[p * kPitch + t];
      }
    }
    __syncthreads(); // the staging area is free for the next tile's operands
  }
  if (abort_s && tid == 0)
    atomicOr(&g_tc5col_fault, 1u);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kCCols)
                 : "memory");
}

} // namespace

cudaError_t launch_tc5_col512_f32(bool fwd, const PassArgs &a, cudaStream_t st) {
  const long long ntiles = (a.total + kCTB - 1) / kCTB;
  if (ntiles <= 0)
    return cudaSuccess;
  auto kern = fwd ? fft_tc5_col512_kernel<true> : fft_tc5_col512_kernel<false>;
  static std::atomic<int> configured_mask{0}; // devices opted in (both directions)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 31)
    return cudaErrorInvalidDevice;
  if (!(configured_mask.load() & (1 << dev))) {
    cudaError_t e = cudaFuncSetAttribute(fft_tc5_col512_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(fft_tc5_col512_kernel<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess)
      return e;
    configured_mask.fetch_or(1 << dev);
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  // two CTAs per SM: 256 TMEM columns each (all 512), 88 KiB of shared memory
  const long long slots = static_cast<long long>(sms) * 2;
  const long long grid = ntiles < slots ? ntiles : slots;
  const char *sv = std::getenv("B200FFT_TC5_STALL_TEST");
  const int stall = (sv != nullptr && sv[0] == '1') ? 1 : 0;
  kern<<<static_cast<unsigned>(grid), kCThreads, kSmemBytes, st>>>(a, stall);
  return cudaGetLastError();
}

// Fault word of the tcgen05 column kernel: returned and cleared (the stream
// of the launches must be synchronised first).
cudaError_t tc5col_take_fault(unsigned *fault) {
  unsigned f = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&f, g_tc5col_fault, sizeof(f));
  if (e != cudaSuccess)
    return e;
  *fault = f;
  if (f) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_tc5col_fault, &zero, sizeof(zero));
  }
  return e;
}

} // namespace b200fft
