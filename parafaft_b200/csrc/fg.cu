// Runtime-generic (Family G) kernels, the twiddle-table kernel and the
// shared-memory size queries used by the planner.
#include <climits>

#include "fft_device.cuh"
#include "launch.hpp"

namespace b200fft {

// ==========================================================================
// Twiddle tables, computed in FP64 and rounded once.
// exp(-2*pi*i*m/n): 4m = q*n + r with integers q (quadrant) and r < n; the
// angle is (pi/2)(q + r/n); the remainder is folded to [0, n/2] so sincospi
// gets an argument in [0, 1/4] that carries no reduction error.
//
// For a power-of-two top length M the table is a pyramid: the M-point table
// T_M[k] = exp(-2*pi*i*k/M), then T_{M/2}, T_{M/4}, ..., T_1, with T_n at
// offset 2M - 2n (2M - 1 entries). T_M alone (offset 0) is what the generic
// kernels index; the specialised kernels read stage twiddles w^p for
// w = exp(-2*pi*i/n) as T_{n/p}[k], contiguous in k. Other lengths get T_M only.
// ==========================================================================
__device__ double2 twiddle_fp64(long long m, long long n) {
  const long long t = 4LL * m;
  const int q = static_cast<int>(t / n);
  const long long r = t - static_cast<long long>(q) * n;
  const bool flip = 2 * r > n;
  const long long rr = flip ? (n - r) : r;
  double s, c;
  sincospi(static_cast<double>(rr) / (2.0 * static_cast<double>(n)), &s, &c);
  if (flip) {
    const double tmp = s;
    s = c;
    c = tmp;
  }
  double cr, ci;
  switch (q & 3) {
  case 0: cr = c; ci = s; break;
  case 1: cr = -s; ci = c; break;
  case 2: cr = -c; ci = -s; break;
  default: cr = s; ci = -c; break;
  }
  return make_double2(cr, -ci);
}

__global__ void twiddle_table_kernel(double2 *t64, float2 *t32, int M, int entries) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= entries)
    return;
  long long n = M, off = 0;
  while (i >= off + n) { // pyramid level of entry i (only for power-of-two M)
    off += n;
    n >>= 1;
  }
  const double2 w = twiddle_fp64(i - off, n);
  if (t64)
    t64[i] = w;
  if (t32)
    t32[i] = make_float2(static_cast<float>(w.x), static_cast<float>(w.y));
}

namespace {

template <typename T, bool COL, int KIND, bool FWD>
cudaError_t launch_g(const GenArgs &g, cudaStream_t st) {
  auto kern = fft_generic_kernel<T, COL, KIND, FWD>;
  const size_t smem = 2ull * g.TB * g.L * sizeof(cvec<T>);
  if (smem > kGenericSmemLimit)
    return cudaErrorInvalidValue;
  // the tile also holds its transforms' offsets in static shared memory, so
  // opt in above 48 KiB of total, not of dynamic, shared memory
  if (smem + kGenStaticSmem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGenericSmemLimit));
    if (e != cudaSuccess)
      return e;
  }
  const long long grid = (g.p.total + g.TB - 1) / g.TB;
  if (grid <= 0)
    return cudaSuccess;
  if (grid > INT_MAX)
    return cudaErrorInvalidConfiguration;
  kern<<<static_cast<unsigned>(grid), kGenThreads, smem, st>>>(g);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_g_t(int kind, bool col, bool fwd, const GenArgs &g,
                       cudaStream_t st) {
  if (kind == KIND_C2C) {
    if (col)
      return fwd ? launch_g<T, true, KIND_C2C, true>(g, st)
                 : launch_g<T, true, KIND_C2C, false>(g, st);
    return fwd ? launch_g<T, false, KIND_C2C, true>(g, st)
               : launch_g<T, false, KIND_C2C, false>(g, st);
  }
  if (kind == KIND_R2C)
    return col ? launch_g<T, true, KIND_R2C, true>(g, st)
               : launch_g<T, false, KIND_R2C, true>(g, st);
  return col ? launch_g<T, true, KIND_C2R, false>(g, st)
             : launch_g<T, false, KIND_C2R, false>(g, st);
}

} // namespace

namespace {
template <typename T, bool COL, int KIND, bool FWD>
cudaError_t launch_gg(const GenArgs *items, const long long *tile_start, int nitems,
                      unsigned long long *queue, size_t smem, int grid, cudaStream_t st) {
  auto kern = fft_generic_group_kernel<T, COL, KIND, FWD>;
  if (smem > kGenericSmemLimit)
    return cudaErrorInvalidValue;
  // the kernel also holds static shared memory (tile offsets, its task), so
  // opt in above 48 KiB of total, not of dynamic, shared memory
  if (smem + kGenStaticSmem + 64 > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kGenericSmemLimit));
    if (e != cudaSuccess)
      return e;
  }
  kern<<<grid, kGenThreads, smem, st>>>(items, tile_start, nitems, queue);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gg_t(int kind, bool col, bool fwd, const GenArgs *items,
                        const long long *tile_start, int nitems, unsigned long long *queue,
                        size_t smem, int grid, cudaStream_t st) {
  if (kind == KIND_C2C) {
    if (col)
      return fwd ? launch_gg<T, true, KIND_C2C, true>(items, tile_start, nitems, queue, smem, grid, st)
                 : launch_gg<T, true, KIND_C2C, false>(items, tile_start, nitems, queue, smem, grid, st);
    return fwd ? launch_gg<T, false, KIND_C2C, true>(items, tile_start, nitems, queue, smem, grid, st)
               : launch_gg<T, false, KIND_C2C, false>(items, tile_start, nitems, queue, smem, grid, st);
  }
  if (kind == KIND_R2C)
    return col ? launch_gg<T, true, KIND_R2C, true>(items, tile_start, nitems, queue, smem, grid, st)
               : launch_gg<T, false, KIND_R2C, true>(items, tile_start, nitems, queue, smem, grid, st);
  return col ? launch_gg<T, true, KIND_C2R, false>(items, tile_start, nitems, queue, smem, grid, st)
             : launch_gg<T, false, KIND_C2R, false>(items, tile_start, nitems, queue, smem, grid, st);
}
} // namespace

cudaError_t launch_generic_group(bool f64, int kind, bool col, bool fwd, const GenArgs *items,
                                 const long long *tile_start, int nitems,
                                 unsigned long long *queue, size_t smem, int grid,
                                 cudaStream_t st) {
  return f64 ? launch_gg_t<double>(kind, col, fwd, items, tile_start, nitems, queue, smem, grid, st)
             : launch_gg_t<float>(kind, col, fwd, items, tile_start, nitems, queue, smem, grid, st);
}

cudaError_t launch_generic(bool f64, int kind, bool col, bool fwd,
                           const GenArgs &g, cudaStream_t st) {
  return f64 ? launch_g_t<double>(kind, col, fwd, g, st)
             : launch_g_t<float>(kind, col, fwd, g, st);
}

size_t generic_smem_bytes(bool f64, int TB, int L) {
  return 2ull * TB * L * (f64 ? sizeof(double2) : sizeof(float2));
}

int twiddle_table_entries(int n) { return is_pow2(n) ? 2 * n - 1 : n; }

cudaError_t launch_twiddle_table(double2 *t64, float2 *t32, int n,
                                 cudaStream_t st) {
  if (n <= 0)
    return cudaErrorInvalidValue;
  const int entries = twiddle_table_entries(n);
  const int threads = 256;
  const int blocks = (entries + threads - 1) / threads;
  twiddle_table_kernel<<<blocks, threads, 0, st>>>(t64, t32, n, entries);
  return cudaGetLastError();
}

} // namespace b200fft
