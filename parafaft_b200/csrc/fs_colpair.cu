// Pair-column C2C kernels, FP32 (tile variant kVariantPair; fft_colpair.cuh).
#include <atomic>
#include <climits>
#include <cstdint>

#include "fft_colpair.cuh"
#include "launch.hpp"

namespace b200fft {

namespace {

template <int L, int NT, int TB, bool FWD, bool VEC>
cudaError_t launch_colpair_one(const PassArgs &a, cudaStream_t st) {
  using K = KP<L, NT, TB, FWD, VEC>;
  auto kern = fft_colpair_kernel<L, NT, TB, FWD, VEC>;
  constexpr size_t smem = K::smem_bytes();
  static std::atomic<int> configured_mask{0}; // devices opted in
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev >= 0 && dev < 31 && !(configured_mask.load() & (1 << dev))) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess)
      return e;
    configured_mask.fetch_or(1 << dev);
  }
  const long long grid = (a.total + TB - 1) / TB;
  if (grid <= 0)
    return cudaSuccess;
  if (grid > INT_MAX)
    return cudaErrorInvalidConfiguration;
  kern<<<static_cast<unsigned>(grid), NT, smem, st>>>(a);
  return cudaGetLastError();
}

template <int L, int NT, int TB>
cudaError_t launch_colpair_l(bool fwd, const PassArgs &a, cudaStream_t st) {
  const bool vec = colpair_vec_ok(a);
  if (fwd)
    return vec ? launch_colpair_one<L, NT, TB, true, true>(a, st)
               : launch_colpair_one<L, NT, TB, true, false>(a, st);
  return vec ? launch_colpair_one<L, NT, TB, false, true>(a, st)
             : launch_colpair_one<L, NT, TB, false, false>(a, st);
}

} // namespace

bool colpair_vec_ok(const PassArgs &a) {
  const auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  return a.idist == 1 && a.odist == 1 && a.batch % 2 == 0 && a.total % 2 == 0 &&
         a.istride % 2 == 0 && a.ostride % 2 == 0 && a.islab % 2 == 0 && a.oslab % 2 == 0 &&
         al(a.in) && al(a.out);
}

bool colpair_length_ok(int L) { return L == 256 || L == 512 || L == 1024; }

cudaError_t launch_colpair_c2c_f32(int L, bool fwd, const PassArgs &a, cudaStream_t st) {
  switch (L) {
  case 256: return launch_colpair_l<256, 512, 32>(fwd, a, st); // 8 points per thread, 256-byte rows
  case 512: return launch_colpair_l<512, 512, 16>(fwd, a, st); // 8 points per thread, 128-byte rows
  case 1024: return launch_colpair_l<1024, 1024, 16>(fwd, a, st); // 8 points, one CTA per SM
  default: return cudaErrorInvalidValue;
  }
}

} // namespace b200fft
