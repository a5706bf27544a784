// Building blocks of the tcgen05 split-precision kernels (fft_tc5.cu,
// fft_tc5col.cu): shared-memory matrix descriptors in the canonical no-swizzle
// layouts, the kind::f16 instruction descriptor, the product, commit and fence
// instructions, a clock-bounded mbarrier wait, TMEM loads, the FP16 hi/lo
// split and power-of-two block scales.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "fft_device.cuh"

namespace b200fft {
namespace tc5 {

BF_D uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

BF_D uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t *>(&h); }

// Packed FP16 hi and lo parts of two FP32 values (a in the low half).
BF_D void split2(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 f = __half22float2(h);
  hi = h2u(h);
  lo = h2u(__floats2half2_rn(a - f.x, b - f.y));
}

// Shared-memory matrix descriptor: no swizzle, version 1 (sm_100).
BF_D uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, FP16 A and B,
// B K-major, A K-major or MN-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_f16(bool a_mn, int M, int N) {
  return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

BF_D void umma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
               : "memory");
}

BF_D void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}

BF_D void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
BF_D void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
BF_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Wait for phase `parity` of the barrier, at most about a second of clock.
// One thread polls (suspended up to 1 us per try); the others wait at the
// CTA barrier that follows, which costs them no issue slots.
BF_D bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done)
                 : "r"(mbar), "r"(parity), "r"(1000u)
                 : "memory");
    if (done)
      return true;
    if (clock64() - t0 > (2ll << 30))
      return false;
  }
}

// 8 consecutive FP32 columns of this thread's TMEM lane (no wait).
BF_D void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i)
    v[i] = __uint_as_float(r[i]);
}
BF_D void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Outputs 8h .. 8h+7 of a step: D = acc_a + acc_b, real columns 8h.., imaginary
// columns 16 + 8h.. of each accumulator.
BF_D void tmem_outputs8(uint32_t tlane, int h, float (&re)[8], float (&im)[8]) {
  float a0[8], a1[8], b0[8], b1[8];
  tmem_ld8(tlane + 8 * h, a0);
  tmem_ld8(tlane + 16 + 8 * h, a1);
  tmem_ld8(tlane + 32 + 8 * h, b0);
  tmem_ld8(tlane + 48 + 8 * h, b1);
  tmem_wait_ld();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    re[i] = a0[i] + b0[i];
    im[i] = a1[i] + b1[i];
  }
}

// Scale 2^(lim - e) for a block whose largest magnitude lies in [2^e, 2^(e+1)),
// clamped so that the scale and its inverse are normal.
BF_D void block_scale(float m, int lim, float &s, float &inv) {
  int sb = 127 + lim + 127 - ((__float_as_int(m) >> 23) & 0xff);
  sb = sb < 1 ? 1 : (sb > 253 ? 253 : sb);
  s = __int_as_float(sb << 23);
  inv = __int_as_float((254 - sb) << 23);
}

// byte offset of element (m, k) (k < 16) in a K-major / MN-major region
BF_D int kmaj(int m, int k) { return (m & 7) * 16 + (k & 7) * 2 + (k >> 3) * 128 + (m >> 3) * 256; }
BF_D int mnmaj(int m, int k) { return (m & 7) * 2 + (k & 7) * 16 + (k >> 3) * 128 + (m >> 3) * 256; }


} // namespace tc5
} // namespace b200fft
