// Dependency-scheduled persistent pass kernel (the group schedule of many
// independent small grids, e.g. a batch of uneven R2C grids). A group takes
// this form when asked (B200FFT_GROUP_SCHEDULE=1); on 256 uneven grids it
// moves about a third of the DRAM bytes of the per-level launches but runs
// slower than them (2.6 vs 2.1 ms), so they stay the default.
//
// A group schedule is a list of passes: pass k of grid g reads what pass k-1
// of the same grid wrote, and grids are independent of one another. Instead
// of one launch per (dependency level, length) with a barrier between levels,
// one persistent kernel walks a device work list of (pass, tile) items in a
// fixed order. Each CTA claims the next item with one atomic; before it
// transforms a tile it waits until every tile of the pass its pass depends on
// has finished (a per-pass completion counter), then it transforms the tile
// with the specialised Family S code of that pass's length, layout, kind and
// direction, and counts the tile as done.
//
// Deadlock freedom: an item is claimed only by a running CTA, items are
// claimed in list order, and a pass is listed after the pass it depends on,
// so every tile a CTA waits for was claimed earlier by a running CTA that
// either finishes it or waits (in turn) only for tiles listed before it.
// Every wait is still bounded by wall-clock time (%globaltimer): when it runs
// out, the CTA sets the fault word, skips the tile's arithmetic (but counts it
// done, so nothing waits on it for ever) and every later wait returns at
// once; the host reports B200FFT_ERR_DEVICE_STATUS at b200fft_group_sync.
//
// Ordering of memory: the finishing CTA's threads write the tile, meet at a
// barrier, then thread 0 fences at GPU scope and increments the counter; a
// waiting CTA's thread 0 reads the counter with acquire semantics at GPU
// scope, fences, and meets its threads at a barrier before they load the
// tile (the pattern of a grid-wide barrier).
//
// Order of the list: pass k of grid g gets the key g + lag*k (lag in grids,
// default 2) and passes are listed by key, so while some grids start their
// first pass, those `lag` grids ahead run their next one. The passes of one
// grid follow each other closely in time, so a grid's intermediate data is
// usually still in L2 when its next pass reads it.
#include <cuda_runtime.h>

#include <climits>

#include "fft_device.cuh"
#include "launch.hpp"

namespace b200fft {

// The specialised tiles the schedule kernel carries: every one runs on
// kSchedThreads threads.
// The lengths are the sides of grids of 2/3/5-smooth sides from 32 to 160
// points (C2C columns) and their R2C half lengths (rows).
#define B2_SCHED_SPECS(X)                                                                \
  X(KIND_R2C, false, true, 16) X(KIND_R2C, false, true, 24) X(KIND_R2C, false, true, 30)  \
  X(KIND_R2C, false, true, 32) X(KIND_R2C, false, true, 40) X(KIND_R2C, false, true, 48)  \
  X(KIND_R2C, false, true, 60) X(KIND_R2C, false, true, 64) X(KIND_R2C, false, true, 80)  \
  X(KIND_C2R, false, false, 16) X(KIND_C2R, false, false, 24)                              \
  X(KIND_C2R, false, false, 30) X(KIND_C2R, false, false, 32)                              \
  X(KIND_C2R, false, false, 40) X(KIND_C2R, false, false, 48)                              \
  X(KIND_C2R, false, false, 60) X(KIND_C2R, false, false, 64)                              \
  X(KIND_C2R, false, false, 80)                                                           \
  X(KIND_C2C, true, true, 32) X(KIND_C2C, true, true, 48) X(KIND_C2C, true, true, 60)     \
  X(KIND_C2C, true, true, 64) X(KIND_C2C, true, true, 80) X(KIND_C2C, true, true, 96)     \
  X(KIND_C2C, true, true, 120) X(KIND_C2C, true, true, 128) X(KIND_C2C, true, true, 160)  \
  X(KIND_C2C, true, false, 32) X(KIND_C2C, true, false, 48)                                \
  X(KIND_C2C, true, false, 60) X(KIND_C2C, true, false, 64)                                \
  X(KIND_C2C, true, false, 80) X(KIND_C2C, true, false, 96)                                \
  X(KIND_C2C, true, false, 120) X(KIND_C2C, true, false, 128)                              \
  X(KIND_C2C, true, false, 160)

namespace {

struct SpecDesc {
  int kind;
  bool col, fwd;
  int L;
};

constexpr SpecDesc kSpecs[] = {
#define B2_SPEC_DESC(K, C, F, LL) SpecDesc{K, C, F, LL},
    B2_SCHED_SPECS(B2_SPEC_DESC)
#undef B2_SPEC_DESC
};
constexpr int kNumSpecs = static_cast<int>(sizeof(kSpecs) / sizeof(kSpecs[0]));

// Column tiles take the half-size tile (at most 16 points per thread), so
// the kernel fits three CTAs per SM (80 registers); full tiles at two CTAs per
// SM ran 3-6% slower on the uneven-grid batch.
constexpr int kSchedMinBlocks = 3;

template <int KIND, bool COL, bool FWD, int L> struct SchedTile {
  static constexpr CfgS cf = cfg_static(8, L, COL, COL ? 1 : 0);
  static_assert(cf.NT == kSchedThreads, "schedule tiles run on kSchedThreads threads");
  using K = KS<float, L, cf.NT, cf.TB, COL, FWD, KIND>;
  static constexpr size_t smem = K::smem_bytes();
  static constexpr int TB = cf.TB;
  static __device__ __forceinline__ void run(const PassArgs &a, unsigned char *sm,
                                             long long tile) {
    K::entry(a, reinterpret_cast<typename K::V *>(sm), tile);
  }
};

constexpr size_t sched_smem_max() {
  size_t m = 0;
#define B2_SPEC_SMEM(K, C, F, LL)                                                        \
  m = SchedTile<K, C, F, LL>::smem > m ? SchedTile<K, C, F, LL>::smem : m;
  B2_SCHED_SPECS(B2_SPEC_SMEM)
#undef B2_SPEC_SMEM
  return m;
}

constexpr size_t kSchedSmem = sched_smem_max();

constexpr int sched_tb(int spec) {
  int i = 0, tb = 0;
#define B2_SPEC_TB(K, C, F, LL)                                                          \
  if (i++ == spec)                                                                       \
    tb = SchedTile<K, C, F, LL>::TB;
  B2_SCHED_SPECS(B2_SPEC_TB)
#undef B2_SPEC_TB
  return tb;
}

__device__ __forceinline__ void sched_dispatch(int spec, const PassArgs &a, unsigned char *sm,
                                               long long tile) {
  int i = 0;
  // a chain of uniform branches: every thread of the CTA takes the same one
#define B2_SPEC_RUN(K, C, F, LL)                                                         \
  if (spec == i++) {                                                                     \
    SchedTile<K, C, F, LL>::run(a, sm, tile);                                            \
    return;                                                                              \
  }
  B2_SCHED_SPECS(B2_SPEC_RUN)
#undef B2_SPEC_RUN
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Wait (thread 0 only) until done[dep] >= need; 1 if the wait gave up.
__device__ int wait_pass(const SchedArgs &s, int dep, unsigned need) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (load_acquire(s.done + dep) >= need)
      return 0;
    if (*reinterpret_cast<volatile unsigned *>(s.fault) != 0)
      return 1;
    if (global_ns() - t0 > s.wait_ns) {
      atomicOr(s.fault, 1u);
      return 1;
    }
    __nanosleep(128);
  }
}

} // namespace

__global__ void __launch_bounds__(kSchedThreads, kSchedMinBlocks)
    fft_sched_kernel(const SchedArgs s) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ long long item_s[2];
  __shared__ int skip_s;
  // Two barriers per tile. Thread 0 claims the next item while the current
  // tile is transformed (the atomic's round trip overlaps the tile) and does
  // the dependency waits; a thread of warp 1 reports each finished tile, so
  // that fence does not hold up thread 0's claim and wait. (Thread 0 must not
  // report its own previous tile after waiting: the next tile may depend on
  // it.)
  if (threadIdx.x == 0)
    item_s[0] = static_cast<long long>(atomicAdd(s.claim, 1ull));
  __syncthreads();
  for (int k = 0;; ++k) {
    const long long it = item_s[k & 1];
    if (it >= s.nitems)
      return; // uniform: every thread read the same claim
    const int2 w = s.items[it];
    const SchedPass &p = s.passes[w.x];
    unsigned long long next = 0;
    if (threadIdx.x == 0) {
      next = atomicAdd(s.claim, 1ull);
      int skip = 0;
      if (p.dep >= 0) {
        skip = wait_pass(s, p.dep, p.need);
        __threadfence();
      }
      skip_s = skip;
    }
    __syncthreads(); // skip_s is set
    if (!skip_s)
      sched_dispatch(p.spec, p.a, smraw, w.y);
    if (threadIdx.x == 0)
      item_s[(k + 1) & 1] = static_cast<long long>(next);
    __syncthreads(); // the tile's stores are issued, shared memory is free
    if (threadIdx.x == 32) {
      __threadfence();
      atomicAdd(s.done + w.x, 1u);
    }
  }
}

int sched_spec_index(int kind, bool col, bool fwd, int L) {
  for (int i = 0; i < kNumSpecs; ++i)
    if (kSpecs[i].kind == kind && kSpecs[i].col == col && kSpecs[i].fwd == fwd &&
        kSpecs[i].L == L)
      return i;
  return -1;
}

int sched_tile_transforms(int spec) { return spec >= 0 && spec < kNumSpecs ? sched_tb(spec) : 0; }

cudaError_t sched_grid(int *grid) {
  static_assert(kSchedSmem * kSchedMinBlocks <= 220 * 1024, "schedule CTAs per SM");
  cudaError_t e = cudaFuncSetAttribute(fft_sched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kSchedSmem));
  if (e != cudaSuccess)
    return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_sched_kernel, kSchedThreads,
                                                    kSchedSmem);
  if (e != cudaSuccess)
    return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess)
    return e;
  *grid = sms * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

cudaError_t launch_sched(const SchedArgs &s, int grid, cudaStream_t st) {
  if (s.nitems <= 0)
    return cudaSuccess;
  const long long g = s.nitems < grid ? s.nitems : grid;
  fft_sched_kernel<<<static_cast<unsigned>(g), kSchedThreads, kSchedSmem, st>>>(s);
  return cudaGetLastError();
}

} // namespace b200fft
