// Instantiation helpers for the specialised (Family S) kernels. Each
// fs_*.cu translation unit includes this file and instantiates one precision
// and kind, so the kernel set compiles in parallel.
#pragma once

#include <atomic>
#include <climits>

#include "fft_device.cuh"
#include "launch.hpp"

namespace b200fft {

template <typename T, int L, bool COL, bool FWD, int KIND, int VAR>
cudaError_t launch_static_one(const PassArgs &a, cudaStream_t st) {
  constexpr CfgS cf = cfg_static(static_cast<int>(sizeof(cvec<T>)), L, COL, VAR);
  using K = KS<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  auto kern = fft_static_kernel<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  constexpr size_t smem = K::smem_bytes();
  if constexpr (smem > 48 * 1024) {
    // The opt-in is per device; setting it again is cheap and idempotent.
    static std::atomic<int> configured_mask{0}; // devices opted in
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 31 && !(configured_mask.load() & (1 << dev))) {
      cudaError_t e = cudaFuncSetAttribute(
          kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess)
        return e;
      configured_mask.fetch_or(1 << dev);
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

inline int sm_count() {
  static std::atomic<int> n[32] = {}; // per device; every thread stores the same value
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 32)
    dev = 0;
  int v = n[dev].load();
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    n[dev].store(v);
  }
  return v;
}

template <typename T, int L, bool FWD>
cudaError_t launch_static_staged(const PassArgs &a, cudaStream_t st) {
  constexpr CfgS cf = cfg_static(static_cast<int>(sizeof(cvec<T>)), L, true, kVariantStaged);
  using K = KS<T, L, cf.NT, cf.TB, true, FWD, KIND_C2C, true>;
  auto kern = fft_static_staged_kernel<T, L, cf.NT, cf.TB, FWD>;
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
  const long long ntiles = (a.total + cf.TB - 1) / cf.TB;
  if (ntiles <= 0)
    return cudaSuccess;
  const int per_sm = smem <= 100 * 1024 ? 2 : 1;
  const long long grid = ntiles < static_cast<long long>(sm_count()) * per_sm
                             ? ntiles
                             : static_cast<long long>(sm_count()) * per_sm;
  kern<<<static_cast<unsigned>(grid), cf.NT, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int L, bool FWD>
cudaError_t launch_static_pipelined(const PassArgs &a, cudaStream_t st) {
  constexpr CfgS cf = cfg_static(static_cast<int>(sizeof(cvec<T>)), L, true, kVariantPipelined);
  using K = KS<T, L, cf.NT, cf.TB, true, FWD, KIND_C2C>;
  auto kern = fft_static_pipelined_kernel<T, L, cf.NT, cf.TB, FWD>;
  constexpr size_t smem = 2 * K::smem_bytes();
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
  const long long ntiles = (a.total + cf.TB - 1) / cf.TB;
  if (ntiles <= 0)
    return cudaSuccess;
  const long long slots = static_cast<long long>(sm_count()) * 2;
  const long long grid = ntiles < slots ? ntiles : slots;
  kern<<<static_cast<unsigned>(grid), cf.NT, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int L, bool COL, bool FWD, int KIND>
cudaError_t launch_static_var(int var, const PassArgs &a, cudaStream_t st) {
  if constexpr (!is_pow2(L)) { // mixed-radix lengths: full tile, or half for columns
    if constexpr (COL)
      if (var == 1)
        return launch_static_one<T, L, COL, FWD, KIND, 1>(a, st);
    return launch_static_one<T, L, COL, FWD, KIND, 0>(a, st);
  }
  if constexpr (COL && KIND == KIND_C2C) {
    if (var == kVariantStaged)
      return launch_static_staged<T, L, FWD>(a, st);
    if (var == kVariantPipelined)
      return launch_static_pipelined<T, L, FWD>(a, st);
  }
  switch (var) {
  case 1: return launch_static_one<T, L, COL, FWD, KIND, 1>(a, st);
  case 2: return launch_static_one<T, L, COL, FWD, KIND, 2>(a, st);
  case 3:
    if constexpr (COL)
      return launch_static_one<T, L, COL, FWD, KIND, 3>(a, st);
    else
      return launch_static_one<T, L, COL, FWD, KIND, 0>(a, st);
  case 5:
    if constexpr (COL)
      return launch_static_one<T, L, COL, FWD, KIND, 5>(a, st);
    else
      return launch_static_one<T, L, COL, FWD, KIND, 0>(a, st);
  case 7:
    if constexpr (COL)
      return launch_static_one<T, L, COL, FWD, KIND, 7>(a, st);
    else
      return launch_static_one<T, L, COL, FWD, KIND, 0>(a, st);
  default: return launch_static_one<T, L, COL, FWD, KIND, 0>(a, st);
  }
}

// Grouped specialised pass (full tile): one CTA per tile of every item.
template <typename T, int L, bool COL, bool FWD, int KIND>
cudaError_t launch_static_group_one(const PassArgs *items, const int2 *tile_map, long long ntiles,
                                    cudaStream_t st) {
  constexpr CfgS cf = cfg_static(static_cast<int>(sizeof(cvec<T>)), L, COL, 0);
  using K = KS<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  auto kern = fft_static_group_kernel<T, L, cf.NT, cf.TB, COL, FWD, KIND>;
  constexpr size_t smem = K::smem_bytes();
  if constexpr (smem > 48 * 1024) {
    static std::atomic<int> configured_mask{0}; // devices opted in
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 31 && !(configured_mask.load() & (1 << dev))) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
      if (e != cudaSuccess)
        return e;
      configured_mask.fetch_or(1 << dev);
    }
  }
  if (ntiles <= 0)
    return cudaSuccess;
  if (ntiles > INT_MAX)
    return cudaErrorInvalidConfiguration;
  kern<<<static_cast<unsigned>(ntiles), cf.NT, smem, st>>>(items, tile_map);
  return cudaGetLastError();
}

#define B2_FG_CASE(LL)                                                         \
  case LL: return launch_static_group_one<T, LL, COL, FWD, KIND>(items, tm, nt, st);

template <typename T, bool COL, bool FWD, int KIND>
cudaError_t launch_static_group_switch(int L, const PassArgs *items, const int2 *tm, long long nt,
                                       cudaStream_t st) {
  switch (L) {
    B2_FG_CASE(2) B2_FG_CASE(4) B2_FG_CASE(8) B2_FG_CASE(16) B2_FG_CASE(32)
    B2_FG_CASE(64) B2_FG_CASE(128) B2_FG_CASE(256) B2_FG_CASE(512)
    B2_FG_CASE(1024) B2_FG_CASE(2048)
    B2_FG_CASE(24) B2_FG_CASE(30) B2_FG_CASE(40) B2_FG_CASE(48) B2_FG_CASE(60)
    B2_FG_CASE(80) B2_FG_CASE(96) B2_FG_CASE(120) B2_FG_CASE(160) B2_FG_CASE(192)
    B2_FG_CASE(384) B2_FG_CASE(768)
  case 4096:
    if constexpr (KIND == KIND_C2C)
      return launch_static_group_one<T, 4096, COL, FWD, KIND>(items, tm, nt, st);
    else
      return cudaErrorInvalidValue;
  default:
    return cudaErrorInvalidValue;
  }
}

#define B2_FS_CASE(LL)                                                         \
  case LL: return launch_static_var<T, LL, COL, FWD, KIND>(var, a, st);

template <typename T, bool COL, bool FWD, int KIND>
cudaError_t launch_static_switch(int L, int var, const PassArgs &a, cudaStream_t st) {
  switch (L) {
    B2_FS_CASE(2) B2_FS_CASE(4) B2_FS_CASE(8) B2_FS_CASE(16) B2_FS_CASE(32)
    B2_FS_CASE(64) B2_FS_CASE(128) B2_FS_CASE(256) B2_FS_CASE(512)
    B2_FS_CASE(1024) B2_FS_CASE(2048)
    B2_FS_CASE(24) B2_FS_CASE(30) B2_FS_CASE(40) B2_FS_CASE(48) B2_FS_CASE(60)
    B2_FS_CASE(80) B2_FS_CASE(96) B2_FS_CASE(120) B2_FS_CASE(160) B2_FS_CASE(192)
    B2_FS_CASE(384) B2_FS_CASE(768)
  case 4096:
    if constexpr (KIND == KIND_C2C)
      return launch_static_var<T, 4096, COL, FWD, KIND>(var, a, st);
    else
      return cudaErrorInvalidValue;
  default:
    return cudaErrorInvalidValue;
  }
}

} // namespace b200fft
