// Instantiation helpers for the specialised (Family S) kernels. Each
// fs_*.cu translation unit includes this file and instantiates one precision
// and kind, so the kernel set compiles in parallel.
#pragma once

#include <climits>

#include "fft_device.cuh"
#include "launch.hpp"

namespace b200fft {

template <typename T, int L, bool COL, bool FWD, int KIND>
cudaError_t launch_static_one(const PassArgs &a, cudaStream_t st) {
  constexpr CfgS cf = cfg_static(static_cast<int>(sizeof(cvec<T>)), L, COL);
  using K = KS<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  auto kern = fft_static_kernel<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  constexpr size_t smem = K::smem_bytes();
  if constexpr (smem > 48 * 1024) {
    // The opt-in is per device; setting it again is cheap and idempotent.
    static int configured_mask = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 31 && !(configured_mask & (1 << dev))) {
      cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess)
        return e;
      configured_mask |= (1 << dev);
    }
  }
  const long long grid = (a.total + cf.TB - 1) / cf.TB;
  if (grid <= 0)
    return cudaSuccess;
  if (grid > INT_MAX)
    return cudaErrorInvalidConfiguration;
  kern<<<static_cast<unsigned>(grid), cf.NT, smem, st>>>(a);
  return cudaGetLastError();
}

#define B2_FS_CASES(T, COL, FWD, KIND)                                          \
  case 2: return launch_static_one<T, 2, COL, FWD, KIND>(a, st);              \
  case 4: return launch_static_one<T, 4, COL, FWD, KIND>(a, st);              \
  case 8: return launch_static_one<T, 8, COL, FWD, KIND>(a, st);              \
  case 16: return launch_static_one<T, 16, COL, FWD, KIND>(a, st);            \
  case 32: return launch_static_one<T, 32, COL, FWD, KIND>(a, st);            \
  case 64: return launch_static_one<T, 64, COL, FWD, KIND>(a, st);            \
  case 128: return launch_static_one<T, 128, COL, FWD, KIND>(a, st);          \
  case 256: return launch_static_one<T, 256, COL, FWD, KIND>(a, st);          \
  case 512: return launch_static_one<T, 512, COL, FWD, KIND>(a, st);          \
  case 1024: return launch_static_one<T, 1024, COL, FWD, KIND>(a, st);        \
  case 2048: return launch_static_one<T, 2048, COL, FWD, KIND>(a, st);

template <typename T, bool COL, bool FWD, int KIND>
cudaError_t launch_static_switch(int L, const PassArgs &a, cudaStream_t st) {
  switch (L) {
    B2_FS_CASES(T, COL, FWD, KIND)
  case 4096:
    if constexpr (KIND == KIND_C2C)
      return launch_static_one<T, 4096, COL, FWD, KIND>(a, st);
    else
      return cudaErrorInvalidValue;
  default:
    return cudaErrorInvalidValue;
  }
}

} // namespace b200fft
