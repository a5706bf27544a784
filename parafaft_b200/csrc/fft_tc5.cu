// Split-precision tensor-core rows on the fifth-generation tensor cores
// (tcgen05): FP32 C2C of length 256, rows (points contiguous).
//
// Same arithmetic as the mma.sync form (fft_tc.cu): 256 = 16 x 16 four-step,
// the DFT-16 blocks as complex matrix products with FP16 hi + lo operands
// (A_lo B_hi + A_hi B_lo + A_hi B_hi) and FP32 accumulation, the two large
// products in separate accumulators, the W256 twiddle in FP32 between steps.
// Here one thread issues each product for the whole CTA:
//   D[128 x 32] = A[128 x 16] * B[16 x 32]   (tcgen05.mma kind::f16, M=128, N=32)
// with A = 128 vectors of 16 points (8 transforms x 16), one k-block for the
// real and one for the imaginary parts, B = the DFT-16 matrix (N = 16 real +
// 16 imaginary outputs), both in shared memory, and D in tensor memory (TMEM).
// Thread r of the CTA owns row r of A and lane r of D: it loads its vector
// from global memory, scales it by a power of two (its own block exponent, no
// cross-thread reduction), splits it and stores its row; after the products it
// reads its 32 outputs back with tcgen05.ld.
//   step 1: row (t, n2) holds x_t[16 n1 + n2], n1 = 0..15 (K-major A);
//   step 2: row (t, k1) holds Y'_t[k1][n2], n2 = 0..15, written by the step-1
//           threads (t, n2) as the MN-major A of the second product, so the
//           corner turn is 16-byte stores;
//   output: thread (t, k1) writes X_t[k1 + 16 k2], k2 = 0..15 (coalesced).
// Operand layouts are the canonical no-swizzle ("interleave") UMMA layouts:
// 8 x 16-byte core matrices, K-major element (m, k) at
// (m%8)*16 + (k%8)*2 + (k/8)*128 + (m/8)*256 bytes, MN-major element (m, k) at
// (m%8)*2 + (k%8)*16 + (k/8)*128 + (m/8)*256 bytes.
//
// Every wait on the MMA-completion barrier is bounded by the clock: past the
// limit the CTA records a fault in a device word (read back by the host at
// b200fft_sync as B200FFT_ERR_DEVICE_STATUS), frees its tensor memory and
// returns.
#include <cuda_fp16.h>

#include <stdint.h>
#include <atomic>
#include <cstdlib>

#include "fft_device.cuh"
#include "launch.hpp"
#include "tc5_common.cuh"

namespace b200fft {
namespace {

using namespace tc5;

__device__ unsigned int g_tc5_fault = 0;

constexpr int kTc5Threads = 128;           // rows of A, lanes of D
constexpr int kTc5TB = 8;                  // transforms per tile
constexpr uint32_t kTc5Cols = 64;          // TMEM: two 32-column accumulators
constexpr int kRegA = 4096;                // bytes of one 128 x 16 FP16 operand
constexpr int kRegB = 1024;                // bytes of one 32 x 16 FP16 operand
// operand regions: 0 hi re, 1 hi im, 2 lo re, 3 lo im

// The six products of one step into accumulators a (hi*hi of the real
// k-block) and b (the rest).
BF_D void issue_step(uint32_t tmem, const unsigned char *A, const unsigned char *B, bool a_mn) {
  const uint32_t id = idesc_f16(a_mn, 128, 32);
  const uint32_t la = 128u, sa = 256u; // K-group and 8-row-group strides (both majors)
  auto ad = [&](int r) { return umma_desc(smem_u32(A + r * kRegA), la, sa); };
  auto bd = [&](int r) { return umma_desc(smem_u32(B + r * kRegB), 128u, 256u); };
  const uint32_t acc_a = tmem, acc_b = tmem + 32;
  umma(acc_b, ad(2), bd(0), id, 0); // lo re * hi
  umma(acc_b, ad(0), bd(2), id, 1); // hi re * lo
  umma(acc_b, ad(3), bd(1), id, 1); // lo im * hi
  umma(acc_b, ad(1), bd(3), id, 1); // hi im * lo
  umma(acc_b, ad(1), bd(1), id, 1); // hi im * hi
  umma(acc_a, ad(0), bd(0), id, 0); // hi re * hi
}

// Eight CTAs per SM (64 registers, 20 KB of shared memory, all 512 TMEM
// columns): the CTAs' load / product / store chains overlap one another.
template <bool FWD>
// stall != 0 (a host-side test switch) issues no products and waits on a
// barrier phase that nothing completes, so the bounded wait runs out and the
// fault path is exercised without any GPU fault.
__global__ void __launch_bounds__(kTc5Threads, 8) fft_tc5_row256_kernel(PassArgs a, int stall) {
  // step 2's operand reuses step 1's: the step-1 products have completed
  // (their barrier phase observed) before it is written
  __shared__ __align__(128) unsigned char sA1[4 * kRegA];
  unsigned char *const sA2 = sA1;
  __shared__ __align__(128) unsigned char sB[4 * kRegB];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_s;
  __shared__ int abort_s;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = tid >> 4, v = tid & 15; // transform of the tile, vector index
  const float2 *tw = static_cast<const float2 *>(a.tw);
  const uint32_t mb = smem_u32(&mbar);

  // ---- set-up: TMEM, barrier, the DFT-16 operand B -------------------------
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_s)),
                 "r"(kTc5Cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_s = 0;
  }
  // B: rows n (outputs: Re k1 = n, Im k1 = n - 16), K = n1; k-block re / im.
  for (int i = tid; i < 32 * 16 * 2; i += kTc5Threads) {
    const int kb = i & 1, k = (i >> 1) & 15, n = i >> 5;
    const int k1 = n & 15;
    const float2 w = __ldg(tw + (2 * 256 - 32) + ((k1 * k) & 15)); // level 16 of the pyramid
    const float c = w.x, s = FWD ? -w.y : w.y;
    const float val = kb == 0 ? (n < 16 ? c : -s) : (n < 16 ? s : c);
    const __half hi = __float2half_rn(val);
    const __half lo = __float2half_rn(val - __half2float(hi));
    const int off = kmaj(n, k);
    *reinterpret_cast<__half *>(sB + (0 + kb) * kRegB + off) = hi;
    *reinterpret_cast<__half *>(sB + (2 + kb) * kRegB + off) = lo;
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_s;
  const uint32_t tlane = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  uint32_t phase = 0;

  const long long ntiles = (a.total + kTc5TB - 1) / kTc5TB;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long b = tile * kTc5TB + t;
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

    // ---- step 1 operand: row (t, n2 = v), K = n1 ---------------------------
    float2 x[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1)
      x[n1] = act ? in[(16 * n1 + v) * a.istride] : make_float2(0.f, 0.f);
    float m = 0.f;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1)
      m = fmaxf(m, fmaxf(fabsf(x[n1].x), fabsf(x[n1].y)));
    float s1, inv1;
    block_scale(m, 14, s1, inv1);
#pragma unroll
    for (int c = 0; c < 2; ++c) { // 8-point chunks of K
      uint32_t hr[4], lr[4], hi[4], li[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float2 p0 = x[8 * c + 2 * q], p1 = x[8 * c + 2 * q + 1];
        split2(p0.x * s1, p1.x * s1, hr[q], lr[q]);
        split2(p0.y * s1, p1.y * s1, hi[q], li[q]);
      }
      const int off = kmaj(tid, 8 * c);
      *reinterpret_cast<uint4 *>(sA1 + 0 * kRegA + off) = make_uint4(hr[0], hr[1], hr[2], hr[3]);
      *reinterpret_cast<uint4 *>(sA1 + 1 * kRegA + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4 *>(sA1 + 2 * kRegA + off) = make_uint4(lr[0], lr[1], lr[2], lr[3]);
      *reinterpret_cast<uint4 *>(sA1 + 3 * kRegA + off) = make_uint4(li[0], li[1], li[2], li[3]);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      if (!stall) {
        issue_step(tmem, sA1, sB, false);
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
    // ---- twiddle, step 2 operand: rows (t, k1), K = n2 (MN-major) ---------
    float2 y[16];
    float m2 = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float re[8], im[8];
      tmem_outputs8(tlane, h, re, im);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k1 = 8 * h + i;
        float2 w = __ldg(tw + ((k1 * v) & 255)); // level 256 at offset 0
        if (!FWD)
          w.y = -w.y;
        y[k1] = cmulw<false>(make_float2(re[i] * inv1, im[i] * inv1), w);
        m2 = fmaxf(m2, fmaxf(fabsf(y[k1].x), fabsf(y[k1].y)));
      }
    }
    // one block exponent per transform: the 16 threads of transform t
#pragma unroll
    for (int o = 1; o < 16; o <<= 1)
      m2 = fmaxf(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    float s2, inv2;
    block_scale(m2, 14, s2, inv2);
#pragma unroll
    for (int c = 0; c < 2; ++c) { // k1 = 8c .. 8c + 7: rows t*16 + k1
      uint32_t hr[4], lr[4], hi[4], li[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float2 p0 = y[8 * c + 2 * q], p1 = y[8 * c + 2 * q + 1];
        split2(p0.x * s2, p1.x * s2, hr[q], lr[q]);
        split2(p0.y * s2, p1.y * s2, hi[q], li[q]);
      }
      const int off = mnmaj(t * 16 + 8 * c, v);
      *reinterpret_cast<uint4 *>(sA2 + 0 * kRegA + off) = make_uint4(hr[0], hr[1], hr[2], hr[3]);
      *reinterpret_cast<uint4 *>(sA2 + 1 * kRegA + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4 *>(sA2 + 2 * kRegA + off) = make_uint4(lr[0], lr[1], lr[2], lr[3]);
      *reinterpret_cast<uint4 *>(sA2 + 3 * kRegA + off) = make_uint4(li[0], li[1], li[2], li[3]);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      issue_step(tmem, sA2, sB, true);
      umma_commit(mb);
      if (!mbar_wait(mb, phase))
        abort_s = 1;
    }
    phase ^= 1;
    fence_after();
    __syncthreads();
    if (abort_s)
      break;
    // ---- output: thread (t, k1 = v) writes X[k1 + 16 k2] -------------------
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float re[8], im[8];
      tmem_outputs8(tlane, h, re, im);
      if (act) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
          out[(v + 16 * (8 * h + i)) * a.ostride] = make_float2(re[i] * inv2, im[i] * inv2);
      }
    }
    fence_before(); // TMEM reads done before the next tile's products
  }
  if (abort_s && tid == 0)
    atomicOr(&g_tc5_fault, 1u);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTc5Cols)
                 : "memory");
}

} // namespace

cudaError_t launch_tc5_row256_f32(bool fwd, const PassArgs &a, cudaStream_t st) {
  const long long ntiles = (a.total + kTc5TB - 1) / kTc5TB;
  if (ntiles <= 0)
    return cudaSuccess;
  static std::atomic<int> per_sm[32] = {}; // per device; every thread stores the same value
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 32)
    return cudaErrorInvalidDevice;
  if (per_sm[dev] == 0) {
    // CTAs per SM from the kernel's registers and shared memory, and its 64
    // of the SM's 512 TMEM columns
    auto kern = fwd ? fft_tc5_row256_kernel<true> : fft_tc5_row256_kernel<false>;
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess)
      return e;
    const int by_regs = fa.numRegs > 0 ? 65536 / (fa.numRegs * kTc5Threads) : 8;
    const int by_smem = static_cast<int>((227 * 1024) / (fa.sharedSizeBytes + 1024));
    int n = by_regs < by_smem ? by_regs : by_smem;
    n = n > 512 / static_cast<int>(kTc5Cols) ? 512 / static_cast<int>(kTc5Cols) : n;
    per_sm[dev] = n < 1 ? 1 : n;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  const long long slots = static_cast<long long>(sms) * per_sm[dev];
  const long long grid = ntiles < slots ? ntiles : slots;
  const char *sv = std::getenv("B200FFT_TC5_STALL_TEST");
  const int stall = (sv != nullptr && sv[0] == '1') ? 1 : 0;
  if (fwd)
    fft_tc5_row256_kernel<true><<<static_cast<unsigned>(grid), kTc5Threads, 0, st>>>(a, stall);
  else
    fft_tc5_row256_kernel<false><<<static_cast<unsigned>(grid), kTc5Threads, 0, st>>>(a, stall);
  return cudaGetLastError();
}

// Fault word of the tcgen05 kernels: returned and cleared (the stream of the
// launches must be synchronised first).
cudaError_t tc5_take_fault(unsigned *fault) {
  unsigned f = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&f, g_tc5_fault, sizeof(f));
  if (e != cudaSuccess)
    return e;
  *fault = f;
  if (f) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_tc5_fault, &zero, sizeof(zero));
  }
  return e;
}

} // namespace b200fft
