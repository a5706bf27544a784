// TMA-fed column passes: FP32 C2C of 256, 512 or 1024 points whose point
// rows are 16-byte aligned (ParaFaFT's first axis, and middle axes of even
// width), and of 256 or 512 points at an odd point stride (the middle axis of
// a padded R2C grid) through a map of double rows (fft_tma_mid_tile_kernel,
// one CTA per tile, and fft_tma_mid_kernel, the ring form, below).
// Both are autotuner candidates (tile variants 8 and 9): on the 512^3 R2C
// step the ring ties the register-direct tile on the aligned first axis
// (0.214 vs 0.212 ms) and the double-row kernels lose on the middle axis
// (0.235 ms one CTA per tile, variant 8; the ring slower; 0.228 ms for the
// register-direct tile: the odd rows' boxes read two extra columns and their
// rows straddle 128-byte lines like plain loads).
//
// A persistent CTA per SM walks its tiles (TB adjacent transforms, 64 KiB)
// through a ring of three shared-memory buffers. Thread 0 fills each buffer
// with bulk tensor copies (cp.async.bulk.tensor, one per 256 point rows, box
// {TB columns, rows, 1 slab} of a 3D map {columns, points, slabs}) that
// complete on the buffer's mbarrier; while the CTA transforms tile t, the
// copies of tiles t+1 and t+2 are in flight, so the load phase of one tile
// overlaps the arithmetic of the previous ones inside the SM instead of
// across co-resident CTAs. The TMA box lands as [point][transform], which is
// the column layout of the Stockham stages (KS::sidx): stage 0 reads its
// points from the buffer, the later stages exchange through the same buffer,
// and the last stage stores to global memory directly.
//
// Every wait on a buffer's barrier is bounded by the clock (about a second);
// past it the CTA sets g_tma_fault, waits (bounded) for the copies it still
// has in flight and returns, and b200fft_sync reports
// B200FFT_ERR_DEVICE_STATUS. B200FFT_TMA_STALL_TEST=1 makes every ring CTA
// skip the copies of its first tile (the one-CTA-per-tile form: tile 0's), so
// that wait runs out (the test of this path: nothing faults, the context stays
// usable).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "fs_launch.cuh"

namespace b200fft {

__device__ unsigned int g_tma_fault = 0;

namespace {

constexpr int kTmaStages = 3;
constexpr int kTmaTileBytes = 64 * 1024; // one tile: 8192 complex64
constexpr int kTmaMaxRows = 256;         // box height limit of a tensor copy
constexpr int kTmaSmem = kTmaStages * kTmaTileBytes;

BF_D uint32_t su32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Phase `parity` of the barrier, at most about a second of clock.
BF_D bool tma_wait(uint32_t mbar, uint32_t parity) {
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

template <int L, int NT, bool FWD>
__global__ void __launch_bounds__(NT, 1)
    fft_tma_col_kernel(const __grid_constant__ CUtensorMap map, const PassArgs a,
                       long long tiles_per_slab, int stall) {
  constexpr int TB = kTmaTileBytes / (L * 8);
  constexpr int ROWS = L < kTmaMaxRows ? L : kTmaMaxRows;
  using K = KS<float, L, NT, TB, true, FWD, KIND_C2C, true>;
  using V = typename K::V;
  static_assert(TB * L * 8 == kTmaTileBytes, "a tile fills one ring buffer");
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long full[kTmaStages];
  __shared__ int abort_flag;
  V *const ring = reinterpret_cast<V *>(smraw);
  const long long slabs = a.total / a.batch;
  const long long ntiles = slabs * tiles_per_slab;
  const long long G = gridDim.x;
  const int tid = threadIdx.x;
  if (static_cast<long long>(blockIdx.x) >= ntiles)
    return;

  // thread 0: the copies of tile `tile` into buffer s, completing on full[s]
  auto issue = [&](long long tile, int s) {
    const long long sl = ntiles == tiles_per_slab ? 0 : tile / tiles_per_slab;
    const int x = static_cast<int>((tile - sl * tiles_per_slab) * TB * 2); // floats
    const uint32_t mb = su32(&full[s]);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                 "r"(kTmaTileBytes)
                 : "memory");
#pragma unroll
    for (int y = 0; y < L; y += ROWS) {
      const uint32_t dst = su32(ring + static_cast<size_t>(s) * L * TB + y * TB);
      asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                   " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                   "l"(reinterpret_cast<uint64_t>(&map)), "r"(x), "r"(y),
                   "r"(static_cast<int>(sl)), "r"(mb)
                   : "memory");
    }
  };

  if (tid == 0) {
    for (int s = 0; s < kTmaStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < kTmaStages; ++s) {
      const long long t = blockIdx.x + s * G;
      if (t < ntiles && !(stall && s == 0))
        issue(t, s);
    }

  typename K::Ctx c;
  c.g = tid / TB;
  c.tb = tid % TB;
  c.tw = reinterpret_cast<const V *>(a.tw);
  c.ist = a.istride;
  c.ost = a.ostride;
  c.gin = nullptr;
  for (long long it = 0;; ++it) {
    const long long tile = blockIdx.x + it * G;
    if (tile >= ntiles)
      break;
    const int s = static_cast<int>(it % kTmaStages);
    const uint32_t parity = static_cast<uint32_t>((it / kTmaStages) & 1);
    if (tid == 0 && !tma_wait(su32(&full[s]), parity)) {
      abort_flag = 1;
      atomicOr(&g_tma_fault, 1u);
    }
    __syncthreads();
    if (abort_flag) {
      // the copies of the later tiles this CTA issued may still be running:
      // wait for them (bounded) before the CTA's shared memory goes away
      if (tid == 0)
        for (int k = 1; k < kTmaStages; ++k) {
          const long long later = it + k;
          if (blockIdx.x + later * G < ntiles)
            tma_wait(su32(&full[later % kTmaStages]),
                     static_cast<uint32_t>((later / kTmaStages) & 1));
        }
      return;
    }
    c.sm = ring + static_cast<size_t>(s) * L * TB;
    const long long sl = ntiles == tiles_per_slab ? 0 : tile / tiles_per_slab;
    const long long w = (tile - sl * tiles_per_slab) * TB + c.tb;
    c.act = w < a.batch;
    c.gout = reinterpret_cast<V *>(a.out) + (c.act ? sl * a.oslab + w * a.odist : 0);
    V v[K::EMAX];
    constexpr int R = K::S.rad[0];
    constexpr int B = L / R;
    constexpr int KB = (B + K::P - 1) / K::P;
    constexpr bool FULL = (B % K::P) == 0;
#pragma unroll
    for (int i = 0; i < KB; ++i) {
      const int j = c.g + K::P * i;
      if (FULL || j < B) {
#pragma unroll
        for (int r = 0; r < R; ++r)
          v[i * R + r] = c.sm[(j + r * B) * TB + c.tb];
      }
    }
    K::template run<0>(c, v);
    __syncthreads(); // every thread is done with buffer s
    if (tid == 0) {
      const long long next = tile + kTmaStages * G;
      if (next < ntiles) {
        // the buffer was last written through the generic proxy (the stage
        // exchanges): order those writes before the async proxy's refill
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(next, s);
      }
    }
  }
}

// Odd point strides (the middle axis of a padded R2C grid: W = N/2+1 complex
// per point row, W odd) break the tensor map's 16-byte stride rule, but two
// neighbouring point rows together are 2W complex = 16W bytes. The pass
// therefore reads the slab through a map of double rows {4W floats, L/2
// double rows, slabs}: point row 2m is columns [0, W) of double row m and
// point row 2m+1 is columns [W, 2W). A tile of TB transforms (columns c0 ..
// c0+TB-1, c0 a multiple of TB) takes two boxes: the even rows at x = c0
// (TB columns, 16-byte aligned since c0 is even) and the odd rows at
// x = W + c0 - 1 (even, so aligned), TB + 2 columns wide; the odd rows' points
// sit one column into that box. Both boxes are L/2 rows high and land side by
// side in one 68 KiB buffer. The W mod TB columns left over at the end of each
// row (one column at W = 257) form remainder tiles after every slab's full
// tiles: TB such columns of different slabs per tile, loaded with plain loads,
// transformed and stored like the others.
template <int L> struct MidGeom {
  static constexpr int TB = kTmaTileBytes / (L * 8);
  static constexpr int HALF = L / 2;                       // double rows per slab
  static constexpr int EVEN_BYTES = TB * HALF * 8;         // box of the even rows
  static constexpr int ODD_W = TB + 2;                     // columns of the odd-row box
  static constexpr int ODD_BYTES = ODD_W * HALF * 8;
  static constexpr int STAGE = EVEN_BYTES + ODD_BYTES;     // one ring buffer
  static constexpr int SMEM = kTmaStages * STAGE;
  static_assert(HALF <= kTmaMaxRows, "one box per parity");
  static_assert(STAGE >= kTmaTileBytes, "the stage exchanges fit in a ring buffer");
  static_assert(EVEN_BYTES % 128 == 0 && STAGE % 128 == 0, "box destinations stay aligned");
};

template <int L, int NT, bool FWD>
__global__ void __launch_bounds__(NT, 1)
    fft_tma_mid_kernel(const __grid_constant__ CUtensorMap map_even,
                       const __grid_constant__ CUtensorMap map_odd, const PassArgs a, int q,
                       long long n_main, long long n_rem, int rem, int stall) {
  using G = MidGeom<L>;
  constexpr int TB = G::TB;
  using K = KS<float, L, NT, TB, true, FWD, KIND_C2C, true>;
  using V = typename K::V;
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long full[kTmaStages];
  __shared__ int abort_flag;
  const long long ntiles = n_main + n_rem;
  const long long GS = gridDim.x;
  const long long W = a.istride;
  const int tid = threadIdx.x;
  if (static_cast<long long>(blockIdx.x) >= ntiles)
    return;

  auto issue = [&](long long tile, int s) {
    const long long sl = tile / q;
    const long long c0 = (tile - sl * q) * TB;
    const uint32_t mb = su32(&full[s]);
    const uint32_t dst = su32(smraw + static_cast<size_t>(s) * G::STAGE);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                 "r"(G::STAGE)
                 : "memory");
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(&map_even)), "r"(static_cast<int>(2 * c0)),
                 "r"(0), "r"(static_cast<int>(sl)), "r"(mb)
                 : "memory");
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst + G::EVEN_BYTES),
                 "l"(reinterpret_cast<uint64_t>(&map_odd)),
                 "r"(static_cast<int>(2 * (W + c0 - 1))), "r"(0), "r"(static_cast<int>(sl)),
                 "r"(mb)
                 : "memory");
  };

  if (tid == 0) {
    for (int s = 0; s < kTmaStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < kTmaStages; ++s) {
      const long long t = blockIdx.x + s * GS;
      if (t < n_main && !(stall && s == 0))
        issue(t, s);
    }

  typename K::Ctx c;
  c.g = tid / TB;
  c.tb = tid % TB;
  c.tw = reinterpret_cast<const V *>(a.tw);
  c.ist = a.istride;
  c.ost = a.ostride;
  c.gin = nullptr;
  constexpr int R = K::S.rad[0];
  constexpr int B = L / R;
  constexpr int KB = (B + K::P - 1) / K::P;
  constexpr bool FULL = (B % K::P) == 0;
  for (long long it = 0;; ++it) {
    const long long tile = blockIdx.x + it * GS;
    if (tile >= ntiles)
      break;
    V v[K::EMAX];
    if (tile < n_main) {
      const int s = static_cast<int>(it % kTmaStages);
      const uint32_t parity = static_cast<uint32_t>((it / kTmaStages) & 1);
      if (tid == 0 && !tma_wait(su32(&full[s]), parity)) {
        abort_flag = 1;
        atomicOr(&g_tma_fault, 1u);
      }
      __syncthreads();
      if (abort_flag) {
        // wait (bounded) for the copies of later tiles still in flight
        if (tid == 0)
          for (int k = 1; k < kTmaStages; ++k) {
            const long long later = it + k;
            if (blockIdx.x + later * GS < n_main)
              tma_wait(su32(&full[later % kTmaStages]),
                       static_cast<uint32_t>((later / kTmaStages) & 1));
          }
        return;
      }
      V *const even = reinterpret_cast<V *>(smraw + static_cast<size_t>(s) * G::STAGE);
      const V *const odd = even + G::EVEN_BYTES / 8 + 1 + c.tb;
      c.sm = even;
      const long long sl = tile / q;
      const long long w = (tile - sl * q) * TB + c.tb;
      c.act = true;
      c.gout = reinterpret_cast<V *>(a.out) + sl * a.oslab + w * a.odist;
#pragma unroll
      for (int i = 0; i < KB; ++i) {
        const int j = c.g + K::P * i;
        if (FULL || j < B) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int n = j + r * B;
            v[i * R + r] = (n & 1) ? odd[(n >> 1) * G::ODD_W] : even[(n >> 1) * TB + c.tb];
          }
        }
      }
      K::template run<0>(c, v);
      __syncthreads(); // every thread is done with buffer s
      if (tid == 0) {
        const long long next = tile + kTmaStages * GS;
        if (next < n_main) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue(next, s);
        }
      }
    } else {
      // remainder tile: columns q*TB .. W-1 of TB slabs; no copy of this CTA
      // is in flight any more (its later tiles are all remainder tiles)
      const long long b = (tile - n_main) * TB + c.tb;
      const long long slabs = a.total / a.batch;
      c.act = b < slabs * rem;
      const long long sl = c.act ? b / rem : 0;
      const long long col = static_cast<long long>(q) * TB + (c.act ? b - sl * rem : 0);
      c.gin = reinterpret_cast<const V *>(a.in) + sl * a.islab + col * a.idist;
      c.gout = reinterpret_cast<V *>(a.out) + sl * a.oslab + col * a.odist;
      c.sm = reinterpret_cast<V *>(smraw);
#pragma unroll
      for (int i = 0; i < KB; ++i) {
        const int j = c.g + K::P * i;
        const bool ok = c.act && (FULL || j < B);
#pragma unroll
        for (int r = 0; r < R; ++r)
          v[i * R + r] = ok ? c.gin[static_cast<long long>(j + r * B) * c.ist] : czero<V>();
      }
      K::template run<0>(c, v);
      __syncthreads();
    }
  }
}

// The same tiles without the ring: one CTA per tile (68 KiB of shared memory,
// two CTAs per SM), the two boxes of its tile waited for on one mbarrier. On
// the 512^3 middle axis this form runs 0.235 ms against 0.29-0.32 ms for the
// ring (one 512-thread CTA per SM leaves the stage barriers uncovered) and
// 0.228 ms for the register-direct tile. The stall test hook skips the copies
// of tile 0 only.
template <int L, int NT, bool FWD>
__global__ void __launch_bounds__(NT, 2)
    fft_tma_mid_tile_kernel(const __grid_constant__ CUtensorMap map_even,
                            const __grid_constant__ CUtensorMap map_odd, const PassArgs a, int q,
                            long long n_main, int rem, int stall) {
  using G = MidGeom<L>;
  constexpr int TB = G::TB;
  using K = KS<float, L, NT, TB, true, FWD, KIND_C2C, true>;
  using V = typename K::V;
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long full;
  __shared__ int abort_flag;
  const long long tile = blockIdx.x;
  const long long W = a.istride;
  const int tid = threadIdx.x;
  typename K::Ctx c;
  c.g = tid / TB;
  c.tb = tid % TB;
  c.tw = reinterpret_cast<const V *>(a.tw);
  c.ist = a.istride;
  c.ost = a.ostride;
  c.gin = nullptr;
  constexpr int R = K::S.rad[0];
  constexpr int B = L / R;
  constexpr int KB = (B + K::P - 1) / K::P;
  constexpr bool FULL = (B % K::P) == 0;
  V v[K::EMAX];
  if (tile < n_main) {
    const long long sl = tile / q;
    const long long c0 = (tile - sl * q) * TB;
    if (tid == 0) {
      const uint32_t mb = su32(&full);
      const uint32_t dst = su32(smraw);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      const bool skip = stall && tile == 0;
      if (!skip) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                     "r"(G::STAGE)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
            "l"(reinterpret_cast<uint64_t>(&map_even)), "r"(static_cast<int>(2 * c0)), "r"(0),
            "r"(static_cast<int>(sl)), "r"(mb)
            : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst + G::EVEN_BYTES),
            "l"(reinterpret_cast<uint64_t>(&map_odd)), "r"(static_cast<int>(2 * (W + c0 - 1))),
            "r"(0), "r"(static_cast<int>(sl)), "r"(mb)
            : "memory");
      }
      abort_flag = 0;
      if (!tma_wait(mb, 0)) {
        abort_flag = 1;
        atomicOr(&g_tma_fault, 1u);
        if (!skip) // copies in flight: wait for them (bounded) before shared memory goes away
          tma_wait(mb, 0);
      }
    }
    __syncthreads();
    if (abort_flag)
      return;
    V *const even = reinterpret_cast<V *>(smraw);
    const V *const odd = even + G::EVEN_BYTES / 8 + 1 + c.tb;
    c.sm = even;
    c.act = true;
    c.gout = reinterpret_cast<V *>(a.out) + sl * a.oslab + (c0 + c.tb) * a.odist;
#pragma unroll
    for (int i = 0; i < KB; ++i) {
      const int j = c.g + K::P * i;
      if (FULL || j < B) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int n = j + r * B;
          v[i * R + r] = (n & 1) ? odd[(n >> 1) * G::ODD_W] : even[(n >> 1) * TB + c.tb];
        }
      }
    }
    K::template run<0>(c, v);
  } else {
    const long long b = (tile - n_main) * TB + c.tb;
    const long long slabs = a.total / a.batch;
    c.act = b < slabs * rem;
    const long long sl = c.act ? b / rem : 0;
    const long long col = static_cast<long long>(q) * TB + (c.act ? b - sl * rem : 0);
    c.gin = reinterpret_cast<const V *>(a.in) + sl * a.islab + col * a.idist;
    c.gout = reinterpret_cast<V *>(a.out) + sl * a.oslab + col * a.odist;
    c.sm = reinterpret_cast<V *>(smraw);
#pragma unroll
    for (int i = 0; i < KB; ++i) {
      const int j = c.g + K::P * i;
      const bool ok = c.act && (FULL || j < B);
#pragma unroll
      for (int r = 0; r < R; ++r)
        v[i * R + r] = ok ? c.gin[static_cast<long long>(j + r * B) * c.ist] : czero<V>();
    }
    K::template run<0>(c, v);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

template <int L, int NT, bool FWD>
cudaError_t launch_tma_t(const PassArgs &a, cudaStream_t st) {
  constexpr int TB = kTmaTileBytes / (L * 8);
  constexpr int ROWS = L < kTmaMaxRows ? L : kTmaMaxRows;
  auto kern = fft_tma_col_kernel<L, NT, FWD>;
  static std::atomic<int> configured_mask{0}; // devices opted in
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 31 && !(configured_mask.load() & (1 << dev))) {
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmem);
    if (e != cudaSuccess)
      return e;
    configured_mask.fetch_or(1 << dev);
  }
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (enc == nullptr)
    return cudaErrorNotSupported;
  const long long slabs = a.total / a.batch;
  // {columns (floats), points, slabs}; strides in bytes for dims 1 and 2
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(2 * a.batch), static_cast<cuuint64_t>(L),
                              static_cast<cuuint64_t>(slabs)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(a.istride) * 8,
                                 static_cast<cuuint64_t>(slabs > 1 ? a.islab
                                                                   : a.istride * L) * 8};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(2 * TB), static_cast<cuuint32_t>(ROWS), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap map;
  const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(a.in),
                         dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const long long tps = (a.batch + TB - 1) / TB;
  const long long ntiles = tps * slabs;
  if (ntiles <= 0)
    return cudaSuccess;
  const long long sms = sm_count();
  const long long grid = ntiles < sms ? ntiles : sms;
  const char *sv = std::getenv("B200FFT_TMA_STALL_TEST");
  const int stall = (sv != nullptr && sv[0] == '1') ? 1 : 0;
  kern<<<static_cast<unsigned>(grid), NT, kTmaSmem, st>>>(map, a, tps, stall);
  return cudaGetLastError();
}

// nt = 512: one CTA per tile (fft_tma_mid_tile_kernel); nt = 1024: persistent
// CTAs through the ring (fft_tma_mid_kernel).
template <int L, int NT, bool FWD>
cudaError_t launch_tma_mid_t(const PassArgs &a, cudaStream_t st) {
  using G = MidGeom<L>;
  constexpr int TB = G::TB;
  constexpr bool kTile = NT == 512;
  auto kern = [] {
    if constexpr (kTile)
      return fft_tma_mid_tile_kernel<L, NT, FWD>;
    else
      return fft_tma_mid_kernel<L, NT, FWD>;
  }();
  static std::atomic<int> configured_mask{0}; // devices opted in
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 31 && !(configured_mask.load() & (1 << dev))) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTile ? G::STAGE : G::SMEM);
    if (e != cudaSuccess)
      return e;
    configured_mask.fetch_or(1 << dev);
  }
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (enc == nullptr)
    return cudaErrorNotSupported;
  const long long W = a.istride;
  const long long slabs = a.total / a.batch;
  // {double-row columns (floats), double rows, slabs}
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(4 * W), static_cast<cuuint64_t>(L / 2),
                              static_cast<cuuint64_t>(slabs)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(16 * W),
                                 static_cast<cuuint64_t>(slabs > 1 ? a.islab : W * L) * 8};
  const cuuint32_t box_even[3] = {static_cast<cuuint32_t>(2 * TB), static_cast<cuuint32_t>(L / 2), 1};
  const cuuint32_t box_odd[3] = {static_cast<cuuint32_t>(2 * G::ODD_W),
                                 static_cast<cuuint32_t>(L / 2), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUtensorMap map_even, map_odd;
  void *base = const_cast<void *>(a.in);
  CUresult r = enc(&map_even, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box_even,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS)
    r = enc(&map_odd, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box_odd, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const int q = static_cast<int>(W / TB);
  const int rem = static_cast<int>(W - static_cast<long long>(q) * TB);
  const long long n_main = slabs * q;
  const long long n_rem = (slabs * rem + TB - 1) / TB;
  const long long ntiles = n_main + n_rem;
  if (ntiles <= 0)
    return cudaSuccess;
  const char *sv = std::getenv("B200FFT_TMA_STALL_TEST");
  const int stall = (sv != nullptr && sv[0] == '1') ? 1 : 0;
  if constexpr (NT == 512) {
    // one CTA per tile
    if (ntiles > INT_MAX)
      return cudaErrorInvalidConfiguration;
    kern<<<static_cast<unsigned>(ntiles), NT, G::STAGE, st>>>(map_even, map_odd, a, q, n_main,
                                                              rem, stall);
  } else {
    // persistent CTAs through the ring
    const long long sms = sm_count();
    const long long grid = ntiles < sms ? ntiles : sms;
    kern<<<static_cast<unsigned>(grid), NT, G::SMEM, st>>>(map_even, map_odd, a, q, n_main, n_rem,
                                                           rem, stall);
  }
  return cudaGetLastError();
}

} // namespace

bool tma_col_ok(int L, const PassArgs &a) {
  if (L != 256 && L != 512 && L != 1024)
    return false;
  if (a.batch <= 0 || a.total % a.batch != 0 || a.idist != 1)
    return false;
  const long long slabs = a.total / a.batch;
  // 16-byte aligned base and strides (the tensor map's rules); x offsets are
  // multiples of 2*TB floats (>= 64 bytes) by construction
  if ((reinterpret_cast<uintptr_t>(a.in) & 15) != 0 || (a.istride & 1) != 0 ||
      a.istride < a.batch)
    return false;
  if (slabs > 1 && ((a.islab & 1) != 0 || a.islab < a.istride * L))
    return false;
  // tensor coordinates are signed 32-bit: the column (in floats) and the slab
  if (2 * a.batch > 0x7fffffffll || slabs > 0x7fffffffll || a.istride * 8 * L >= (1ll << 40) ||
      (slabs > 1 && a.islab * 8 >= (1ll << 40)))
    return false;
  return encode_fn() != nullptr;
}

// Odd point strides through the double-row map: FP32 256/512-point columns
// whose transforms are all the columns of their point rows (batch == stride,
// unit distance), the stride odd, 16-byte aligned base and slab distance.
bool tma_mid_ok(int L, const PassArgs &a) {
  if (L != 256 && L != 512)
    return false;
  const long long W = a.istride;
  if (a.batch <= 0 || a.batch != W || (W & 1) == 0 || a.idist != 1 || a.total % a.batch != 0)
    return false;
  const long long TB = kTmaTileBytes / (L * 8);
  if (W < TB + 2) // at least one full tile whose odd-row box stays in its double row
    return false;
  const long long slabs = a.total / a.batch;
  if ((reinterpret_cast<uintptr_t>(a.in) & 15) != 0)
    return false;
  if (slabs > 1 && ((a.islab & 1) != 0 || a.islab < W * L))
    return false;
  if (4 * W > 0x7fffffffll || slabs > 0x7fffffffll || 16 * W >= (1ll << 40) ||
      (slabs > 1 && a.islab * 8 >= (1ll << 40)))
    return false;
  return encode_fn() != nullptr;
}

cudaError_t launch_tma_mid_c2c_f32(int L, bool fwd, int nt, const PassArgs &a, cudaStream_t st) {
#define B2_TMAM(LL)                                                                  \
  case LL:                                                                           \
    if (nt == 1024)                                                                  \
      return fwd ? launch_tma_mid_t<LL, 1024, true>(a, st)                            \
                 : launch_tma_mid_t<LL, 1024, false>(a, st);                          \
    return fwd ? launch_tma_mid_t<LL, 512, true>(a, st) : launch_tma_mid_t<LL, 512, false>(a, st);
  switch (L) {
    B2_TMAM(256)
    B2_TMAM(512)
  default:
    return cudaErrorInvalidValue;
  }
#undef B2_TMAM
}

// FP32 column C2C pass through the TMA ring (nt = 512 or 1024 threads per
// CTA); the caller checks tma_col_ok first.
cudaError_t launch_tma_col_c2c_f32(int L, bool fwd, int nt, const PassArgs &a,
                                   cudaStream_t st) {
#define B2_TMA(LL)                                                                   \
  case LL:                                                                           \
    if (nt == 1024)                                                                  \
      return fwd ? launch_tma_t<LL, 1024, true>(a, st) : launch_tma_t<LL, 1024, false>(a, st); \
    return fwd ? launch_tma_t<LL, 512, true>(a, st) : launch_tma_t<LL, 512, false>(a, st);
  switch (L) {
    B2_TMA(256)
    B2_TMA(512)
    B2_TMA(1024)
  default:
    return cudaErrorInvalidValue;
  }
#undef B2_TMA
}

// Fault word of the TMA column kernels: returned and cleared (the stream of
// the launches must be synchronised first).
cudaError_t tma_take_fault(unsigned *fault) {
  unsigned f = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&f, g_tma_fault, sizeof(f));
  if (e != cudaSuccess)
    return e;
  *fault = f;
  if (f) {
    const unsigned zero = 0;
    e = cudaMemcpyToSymbol(g_tma_fault, &zero, sizeof(zero));
  }
  return e;
}

} // namespace b200fft
