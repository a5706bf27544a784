// Host runtime and C ABI of the B200 transform engine (include/b200fft.h).
//
// A handle is one ParaFaFT backend object (backend/fft_backend.hpp:45-196):
// it owns a stream, the per-stage C2C plans, the in-place R2C/C2R plans and
// the twiddle tables, and it holds back two kinds of work so that it can fuse
// them:
//   * a device-to-device memcpy (ParaFaFT's single-rank exchange_local,
//     parafaft_common.hpp:467-543) whose destination the next transform reads
//     is folded into that transform: the kernel reads the copy's source and
//     writes the destination;
//   * execute_stage calls of a middle-axis stage on consecutive slices (the
//     leading-dimension loop, parafaft_c2c.hpp:875-896,
//     parafaft_r2c.hpp:1224-1244) accumulate into one launch that starts when
//     the loop's last slice arrives.
// The number of slices of such a loop is inferred from the plans: a stage plan
// of ParaFaFT's middle-axis form (stride == batch, dist == 1) whose
// length*batch divides the element count of the full stage buffer (the largest
// length*batch over all plans; (N/2+1)*batch for R2C) covers total/(length*batch)
// slices.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/b200fft.h"
#include "fft_common.hpp"
#include "launch.hpp"

using namespace b200fft;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(B200FFT_ERR_CUDA, std::string("CUDA error in ") + what + ": " +
                                    cudaGetErrorString(e));
}

#define B2_TRY(expr)                                                           \
  do {                                                                         \
    int rc_ = (expr);                                                          \
    if (rc_ != B200FFT_SUCCESS)                                                \
      return rc_;                                                              \
  } while (0)

bool env_flag(const char *name) {
  const char *v = std::getenv(name);
  return v != nullptr && v[0] != '\0' && v[0] != '0';
}

// Kernel choice of a plan.
struct Choice {
  int family = 0; // 0 static, 1 generic, 2 split-precision tensor core (mma.sync),
                  // 3 split-precision tensor core on tcgen05
  bool col = false;
  int L = 0;      // complex points of the stage loop
  int tlen = 0;   // twiddle table length
  int TB = 0, NT = 0;
  int esize = 8;   // bytes per complex element
  int variant = 0; // tile-shape candidate of a specialised kernel
  GenArgs gen{};
};

struct Plan {
  bool valid = false;
  int kind = KIND_C2C;
  int len = 0;
  long long batch = 0, stride = 0, dist = 0;
  Choice ch;
};

struct HeldCopy {
  bool active = false;
  char *dst = nullptr;
  const char *src = nullptr;
  size_t bytes = 0;
};

// A held device-to-device 2D copy (ParaFaFT_R2C::copy_real_to_padded,
// parafaft_r2c.hpp:804-822): fused into the R2C pass that follows it.
struct HeldCopy2D {
  bool active = false;
  char *dst = nullptr;
  const char *src = nullptr;
  size_t dpitch = 0, spitch = 0, width = 0, height = 0;
};

// An operation recorded while the handle is inside a group.
struct RecOp {
  enum { PASS = 0, COPY = 1, COPY2D = 2 };
  int type = PASS;
  Plan plan;
  int dir = 0;
  const void *in = nullptr;
  void *out = nullptr;
  const void *tw = nullptr;
  long long slabs = 1, slab = 0;
  void *dst = nullptr;
  const void *src = nullptr;
  size_t bytes = 0, dpitch = 0, spitch = 0, width = 0, height = 0;
};

struct HeldRun {
  bool active = false;
  int stage = -1;
  int dir = 0;
  char *out0 = nullptr;
  long long count = 0;
  long long lead = 1;
  size_t slab_bytes = 0;
  bool fused = false;
};

// Factor a length for the generic kernel: 8s, one 4 or 2, 5s, 3s, then other
// primes up to kGenMaxPrime. Returns false for an unsupported length.
bool gen_schedule(int L, int *rad, int *nst) {
  int m = L, k = 0;
  auto push = [&](int r) -> bool {
    if (k >= kGenMaxStages)
      return false;
    rad[k++] = r;
    m /= r;
    return true;
  };
  while (m % 8 == 0)
    if (!push(8)) return false;
  if (m % 4 == 0 && !push(4)) return false;
  if (m % 2 == 0 && !push(2)) return false;
  while (m % 5 == 0)
    if (!push(5)) return false;
  while (m % 3 == 0)
    if (!push(3)) return false;
  for (int p = 7; p <= kGenMaxPrime && m > 1; p += 2) {
    while (m % p == 0)
      if (!push(p)) return false;
  }
  *nst = k;
  return m == 1;
}

int ilog2(int x) {
  int l = 0;
  while ((1 << l) < x)
    ++l;
  return l;
}

// Tile-shape candidate used without autotuning. Column passes whose points
// lie 4 MiB or more apart (the first axis of large grids) read wider
// contiguous segments per point row with the wide tile; other FP32 columns of
// 512 or more points use the 512-thread full tile; everything else the full
// tile (measured on the 512^3 and 1024^3 passes).
int default_variant(int csize, int L, bool col, long long stride) {
  if (col && !is_pow2(L))
    // FP32 mixed-length columns of up to 256 points: the half tile (still >= 16
    // transforms; 60/80/120/160 points 6-12% faster as single plans; grouped
    // launches keep the full tile, where the half tile was slower)
    return (csize == 8 && L <= 256) ? 1 : 0;
  if (col) {
    // 2048+ points: the wide tile at any stride (its 2-8 transforms per tile
    // still give 32-64-byte row segments, the full tile's half that: FP32 and
    // FP64 2048-point columns at a 1 MiB stride 2.0 -> 3.4 TB/s)
    if (L >= 2048)
      return 3;
    // 1024 points: the wide tile once point rows are 4 MiB or more apart
    // (first axes: FP32 4.3 vs 2.9 TB/s, FP64 3.9 vs 3.0), else the full tile
    // (FP32: 32 points per thread, two 32-point stages)
    if (L == 1024)
      return stride * csize >= (4ll << 20) ? 3 : 0;
    // FP32 columns of 128-512 points: 512-thread full tiles, two CTAs per SM
    // (at 4 MiB strides 128/256 points 6.1 TB/s vs 4.5-5.0 for the other tiles)
    if (csize == 8 && L >= 128)
      return 5;
    // FP64 columns of 512 points or fewer: the full tile at any stride
    // (256 points at a 4 MiB stride 6.4 vs 4.7 TB/s for the wide tile)
    return 0;
  }
  // rows of 256 points (FP32, FP64): twice the points per thread (16), so the
  // radix-16 schedule needs two stages instead of three. 512-point FP32 rows
  // keep the full tile (16 points, three CTAs per SM): 0.35 vs 0.36-0.43 ms
  // for 512^3 C2C rows at 32 points per thread.
  if (L == 256)
    return 1;
  return 0;
}

// Choose the kernel for a plan. kind: KIND_C2C/R2C/C2R. `variant` >= 0 asks
// for that tile-shape candidate of the specialised kernel (else the default).
// split_tc asks for the split-precision tensor-core kernels where they exist
// (FP32 C2C of length 256, 512 or 1024).
int choose_kernel(int prec, int kind, int len, long long batch, long long stride,
                  long long dist, bool force_generic, Choice *out, int variant = -1,
                  bool split_tc = false) {
  const int csize = prec == B200FFT_F64 ? 16 : 8;
  Choice ch;
  ch.esize = csize;
  int L = len;
  bool odd = false;
  if (kind == KIND_C2C) {
    ch.col = dist < stride;
    ch.tlen = len;
  } else {
    odd = (len % 2) != 0;
    L = odd ? len : len / 2;
    ch.col = false;
    ch.tlen = len;
  }
  ch.L = L;
  if (split_tc && !force_generic && prec == B200FFT_F32 && kind == KIND_C2C &&
      tc_length_ok(L)) {
    ch.family = 2;
    ch.variant = 0;
    ch.TB = ch.col ? 16 : 4;
    ch.NT = ch.col ? (L == 1024 ? 512 : 256) : 128;
    // 256-point rows run on the tcgen05 kernel (faster than the mma.sync one);
    // B200FFT_TC_FORM=mma keeps them on mma.sync
    const char *form = std::getenv("B200FFT_TC_FORM");
    if (!ch.col && L == 256 && !(form != nullptr && std::string(form) == "mma")) {
      ch.family = 3;
      ch.TB = 8;
      ch.NT = 128;
    }
    // 512-point columns: the mma.sync kernel by default; B200FFT_TC_FORM=tc5
    // runs them on the tcgen05 column kernel (family 5: correct, but its
    // tiles are not pipelined and it ran 0.44-0.49 ms against 0.31-0.43 ms
    // for the mma.sync form on the 512^3 column passes)
    if (ch.col && L == 512 && form != nullptr && std::string(form) == "tc5") {
      ch.family = 5;
      ch.TB = 16;
      ch.NT = 512;
    }
    *out = ch;
    return B200FFT_SUCCESS;
  }
  const bool static_ok =
      !force_generic && static_length_ok(L) &&
      (kind == KIND_C2C || (!odd && stride == 1 && dist % 2 == 0 && L <= 2048));
  if (static_ok) {
    int var = default_variant(csize, L, ch.col, stride);
    if (const char *v = std::getenv("B200FFT_VARIANT")) {
      char *end = nullptr;
      const long ev = std::strtol(v, &end, 10);
      if (end != v && *end == '\0' && ev >= 0 && ev < kStaticVariants)
        var = static_cast<int>(ev);
    }
    if (variant >= 0 && variant < kStaticVariants)
      var = variant;
    if (!is_pow2(L) && !(ch.col && var == 1))
      var = 0; // mixed-radix lengths: the full tile, or the half tile for columns
    if (var == kVariantPair &&
        !(ch.col && kind == KIND_C2C && csize == 8 && colpair_length_ok(L)))
      var = default_variant(csize, L, ch.col, stride); // the pair tile does not apply
    const CfgS c = cfg_static(csize, L, ch.col, var);
    ch.variant = var;
    ch.family = 0;
    ch.TB = c.TB;
    ch.NT = c.NT;
    *out = ch;
    return B200FFT_SUCCESS;
  }
  // generic
  GenArgs &g = ch.gen;
  std::memset(&g, 0, sizeof(g));
  if (!gen_schedule(L, g.rad, &g.nst))
    return fail(B200FFT_ERR_UNSUPPORTED,
                "b200fft: length " + std::to_string(len) +
                    " has a prime factor above " + std::to_string(kGenMaxPrime) +
                    "; no kernel for it");
  const size_t one = 2ull * L * csize;
  if (one > kGenericSmemLimit)
    return fail(B200FFT_ERR_UNSUPPORTED,
                "b200fft: length " + std::to_string(len) +
                    " exceeds the single-pass limit of the generic kernel");
  int TB = 1;
  const size_t target = 48 * 1024;
  while (TB < kGenMaxTB && one * (2 * TB) <= target)
    TB *= 2;
  g.L = L;
  g.nreal = kind == KIND_C2C ? 0 : len;
  g.odd = odd ? 1 : 0;
  if (kind == KIND_C2C)
    g.lout = L;
  else if (kind == KIND_R2C)
    g.lout = odd ? len / 2 + 1 : L + 1;
  else
    g.lout = odd ? len : L;
  g.TB = TB;
  g.logTB = ilog2(TB);
  g.tscale = (kind != KIND_C2C && !odd) ? 2 : 1;
  int p = 1;
  for (int s = 0; s < g.nst; ++s) {
    g.nsv[s] = p;
    g.ns[s] = make_fastdiv(static_cast<uint32_t>(p));
    g.bq[s] = make_fastdiv(static_cast<uint32_t>(L / g.rad[s]));
    p *= g.rad[s];
  }
  g.Ldiv = make_fastdiv(static_cast<uint32_t>(L));
  g.Loutdiv = make_fastdiv(static_cast<uint32_t>(g.lout));
  ch.family = 1;
  ch.TB = TB;
  ch.NT = kGenThreads;
  *out = ch;
  return B200FFT_SUCCESS;
}

std::string describe_choice(const Choice &ch, int kind) {
  char buf[256];
  std::string rad;
  if (ch.family >= 2) {
    rad = (ch.L > 256 ? std::to_string(ch.L / 256) + "x" : std::string()) + "16x16";
  } else if (ch.family == 0) {
    int r[24] = {}, rest = 1;
    const int n = static_schedule(ch.L, radix_cap(ch.esize, ch.L, ch.TB, ch.NT),
                                  ch.col ? 0 : even_row_threads(ch.L, ch.esize, ch.NT / ch.TB),
                                  r, rest);
    for (int i = 0; i < n; ++i)
      rad += (i ? "x" : "") + std::to_string(r[i]);
  } else {
    for (int s = 0; s < ch.gen.nst; ++s)
      rad += (s ? "x" : "") + std::to_string(ch.gen.rad[s]);
  }
  if (rad.empty())
    rad = "1";
  const char *kn = kind == KIND_C2C ? "c2c" : (kind == KIND_R2C ? "r2c" : "c2r");
  std::snprintf(buf, sizeof(buf), "%s %s L=%d %s tb=%d nt=%d radices=%s var=%d",
                ch.family == 0   ? "static"
                : ch.family == 2 ? "split-tc"
                : ch.family == 3 ? "split-tc5"
                : ch.family == 5 ? "split-tc5col"
                                 : "generic",
                kn, ch.L,
                ch.col ? "col" : "row", ch.TB, ch.NT, rad.c_str(), ch.variant);
  return buf;
}

std::mutex g_alloc_mu;

} // namespace

namespace b200fft {
// Lets other translation units of the library report through
// b200fft_last_error().
void set_error_text(const std::string &msg) { g_err = msg; }
} // namespace b200fft

struct b200fft_handle_s {
  int prec = B200FFT_F32;
  int rsize = 4; // bytes of FloatType
  int nstages = 0;
  int plan_flag = 0;
  unsigned flags = 0;
  bool record_only = false;
  bool defer = true;
  bool force_generic = false;
  bool split_tc = false; // split-precision tensor-core kernels where they exist
  bool used_tc5 = false; // launched a tcgen05 kernel (check its fault word at sync)
  bool used_tma = false; // launched a TMA column kernel (check its fault word at sync)
  bool last_tma = false; // the last transform launch ran the TMA column kernel
  int device = -1;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<Plan> stages;
  Plan r2c, c2r;
  std::map<int, void *> tables;
  HeldCopy copy;
  HeldCopy2D pad;
  HeldRun run;
  b200fft_stats stats{};
  std::deque<b200fft_launch_record> log;
  // per-launch timing
  bool profiling = false;
  struct Timed {
    size_t seq;
    cudaEvent_t a, b;
  };
  std::deque<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  size_t seq = 0;        // sequence number of the next log record
  size_t log_base = 0;   // sequence number of log.front()
  // planning buffer for timing candidates (Measure/Patient plans)
  void *work = nullptr;
  size_t work_bytes = 0;
  // group membership (b200fft_group_*)
  b200fft_group_s *group = nullptr;
  bool recording = false;
  std::vector<RecOp> recs;

  size_t csize() const { return 2 * static_cast<size_t>(rsize); }
};

namespace {

struct GroupStep {
  // SINGLE: a level's only pass of its (length, layout, kind, direction): it
  // runs the plan's own kernel choice (tile variant, TMA or tensor-core form)
  // on the group's stream rather than the grouped kernel's default tile.
  enum { PASSES = 0, COPY = 1, COPY2D = 2, STATIC = 3, SINGLE = 4 };
  int type = PASSES;
  // grouped pass: generic kernel (PASSES, items) or specialised kernel of
  // length L (STATIC, sitems)
  bool f64 = false, col = false, fwd = true;
  int kind = KIND_C2C;
  int L = 0;
  std::vector<GenArgs> items;
  std::vector<PassArgs> sitems;
  std::vector<long long> tile_start;
  int2 *d_tile_map = nullptr; // STATIC: (item, tile within the item) per tile
  GenArgs *d_items = nullptr;
  PassArgs *d_sitems = nullptr;
  long long *d_tile_start = nullptr;
  size_t smem = 0;
  int grid = 0;
  int queue = 0;
  long long bytes = 0;
  // copy
  RecOp op;
  int level = 0; // dependency level (the level's steps are independent)
  int chain = 0; // chain of grids the step belongs to (chains are independent)
  // SINGLE (and the first item of a STATIC step)
  b200fft_handle_s *h = nullptr;
  Plan plan;
  int dir = 0;
  PassArgs pa{};
};

} // namespace

// Streams a level of a group schedule spreads its independent steps over.
constexpr int kGroupStreams = 8;

struct b200fft_group_s {
  std::vector<b200fft_handle_s *> handles;
  cudaStream_t stream = nullptr;
  bool record_only = false;
  bool recording = false;
  std::vector<GroupStep> steps;
  unsigned long long *d_queues = nullptr;
  int nqueues = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  b200fft_stats stats{};
  // The steps of one level run side by side: step i of a level on lane
  // i % lanes, forked from and joined back into the chain's first lane by
  // events around the level. Independent chains of grids
  // (B200FFT_GROUP_CHAINS): chain c's levels run on lanes[c] (lanes[0][0] is
  // the group's stream), forked from the group's stream at the start and
  // joined back at the end, so one chain's level tails overlap the other
  // chains' work.
  int chains = 1;
  std::vector<std::vector<cudaStream_t>> lanes;      // [chain][lane]
  std::vector<std::vector<cudaEvent_t>> lane_done;   // [chain][lane]
  std::vector<cudaEvent_t> chain_start;              // [chain] level fork
  cudaEvent_t fork_ev = nullptr;
  // The dependency-scheduled form (fft_sched.cu, B200FFT_GROUP_SCHEDULE=1):
  // when every recorded pass has a tile in the schedule kernel, the whole
  // schedule is one persistent launch over a (pass, tile) work list instead
  // of the level steps.
  bool sched = false;
  std::vector<SchedPass> spasses;
  std::vector<int2> sorder;
  SchedPass *d_spasses = nullptr;
  int2 *d_sorder = nullptr;
  unsigned *d_sdone = nullptr;              // per-pass tile counters
  unsigned long long *d_sclaim = nullptr;   // next work item
  unsigned *d_sfault = nullptr;             // a wait ran out of time
  int sgrid = 0;
  long long sbytes = 0;
  unsigned long long swait_ns = 1000000000ull;
};

namespace {

using H = b200fft_handle_s;

void push_log(H *h, b200fft_launch_record r) {
  r.ms = -1.0;
  h->log.push_back(r);
  h->seq++;
  if (h->log.size() > 4096) {
    h->log.pop_front();
    h->log_base++;
  }
}

cudaEvent_t take_event(H *h) {
  if (!h->event_pool.empty()) {
    cudaEvent_t e = h->event_pool.back();
    h->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

// Bracket the next device operation with events when profiling.
struct ProfileScope {
  H *h;
  cudaEvent_t a = nullptr;
  explicit ProfileScope(H *hh) : h(hh) {
    if (h->profiling && !h->record_only) {
      a = take_event(h);
      if (a)
        cudaEventRecord(a, h->stream);
    }
  }
  // call after push_log of the operation's record
  void done() {
    if (!a)
      return;
    cudaEvent_t b = take_event(h);
    if (!b) {
      h->event_pool.push_back(a);
      return;
    }
    cudaEventRecord(b, h->stream);
    h->timed.push_back({h->seq - 1, a, b});
    a = nullptr;
  }
};

// Resolve pending timings into the log (blocks on the events).
void resolve_timings(H *h) {
  while (!h->timed.empty()) {
    auto t = h->timed.front();
    h->timed.pop_front();
    float ms = -1.0f;
    if (cudaEventSynchronize(t.b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      if (t.seq >= h->log_base && t.seq - h->log_base < h->log.size())
        h->log[t.seq - h->log_base].ms = ms;
    } else {
      cudaGetLastError();
    }
    h->event_pool.push_back(t.a);
    h->event_pool.push_back(t.b);
  }
}

int get_table(H *h, int n, const void **out) {
  if (h->record_only) {
    *out = nullptr;
    return B200FFT_SUCCESS;
  }
  auto it = h->tables.find(n);
  if (it != h->tables.end()) {
    *out = it->second;
    return B200FFT_SUCCESS;
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, static_cast<size_t>(twiddle_table_entries(n)) * h->csize());
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMalloc (twiddle table)");
  if (h->prec == B200FFT_F64)
    e = launch_twiddle_table(static_cast<double2 *>(p), nullptr, n, h->stream);
  else
    e = launch_twiddle_table(nullptr, static_cast<float2 *>(p), n, h->stream);
  if (e != cudaSuccess) {
    cudaFree(p);
    return cuda_fail(e, "twiddle table kernel");
  }
  h->tables[n] = p;
  *out = p;
  return B200FFT_SUCCESS;
}

// Elements (complex) in the largest stage buffer any plan covers.
long long full_elems(const H *h) {
  long long t = 0;
  for (const Plan &p : h->stages)
    if (p.valid)
      t = std::max(t, static_cast<long long>(p.len) * p.batch);
  if (h->r2c.valid)
    t = std::max(t, static_cast<long long>(h->r2c.len / 2 + 1) * h->r2c.batch);
  if (h->c2r.valid)
    t = std::max(t, static_cast<long long>(h->c2r.len / 2 + 1) * h->c2r.batch);
  return t;
}

long long infer_lead(const H *h, const Plan &p) {
  if (!h->defer)
    return 1;
  if (p.dist != 1 || p.stride != p.batch)
    return 1;
  const long long slab = static_cast<long long>(p.len) * p.batch;
  const long long t = full_elems(h);
  if (slab <= 0 || t <= slab || t % slab != 0)
    return 1;
  return t / slab;
}

size_t c2c_span_bytes(const H *h, const Plan &p) {
  const long long e = static_cast<long long>(p.len - 1) * p.stride +
                      (p.batch - 1) * p.dist + 1;
  return static_cast<size_t>(e) * h->csize();
}

size_t real_span_bytes(const H *h, const Plan &p) {
  // reals touched: input (len-1)*stride+1, complex output 2*(len/2)*stride+2
  const long long in_r = static_cast<long long>(p.len - 1) * p.stride + 1;
  const long long out_r = 2LL * (p.len / 2) * p.stride + 2;
  const long long e = (p.batch - 1) * p.dist + std::max(in_r, out_r);
  return static_cast<size_t>(e) * h->rsize;
}

bool overlaps(const char *a, size_t na, const char *b, size_t nb) {
  return a < b + nb && b < a + na;
}

int issue_copy(H *h, void *dst, const void *src, size_t bytes) {
  if (bytes == 0 || dst == src)
    return B200FFT_SUCCESS;
  if (h->recording) {
    RecOp op;
    op.type = RecOp::COPY;
    op.dst = dst;
    op.src = src;
    op.bytes = bytes;
    h->recs.push_back(op);
    return B200FFT_SUCCESS;
  }
  h->stats.copies_issued++;
  h->stats.bytes_copied += bytes;
  b200fft_launch_record r{};
  r.kind = 3;
  r.stage = -1;
  r.family = -1;
  r.bytes = static_cast<long long>(bytes);
  if (h->record_only) {
    push_log(h, r);
    return B200FFT_SUCCESS;
  }
  ProfileScope ps(h);
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, h->stream);
  push_log(h, r);
  ps.done();
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMemcpyAsync");
  return B200FFT_SUCCESS;
}

int flush_copy(H *h) {
  if (!h->copy.active)
    return B200FFT_SUCCESS;
  h->copy.active = false;
  return issue_copy(h, h->copy.dst, h->copy.src, h->copy.bytes);
}

int issue_copy2d(H *h, void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                 size_t height) {
  h->stats.copies_issued++;
  h->stats.bytes_copied += width * height;
  b200fft_launch_record r{};
  r.kind = 3;
  r.stage = -1;
  r.family = -1;
  r.bytes = static_cast<long long>(width * height);
  if (h->record_only) {
    push_log(h, r);
    return B200FFT_SUCCESS;
  }
  ProfileScope ps(h);
  cudaError_t e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height,
                                    cudaMemcpyDefault, h->stream);
  push_log(h, r);
  ps.done();
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaMemcpy2DAsync");
  return B200FFT_SUCCESS;
}

int flush_pad(H *h) {
  if (!h->pad.active)
    return B200FFT_SUCCESS;
  h->pad.active = false;
  const HeldCopy2D c = h->pad;
  return issue_copy2d(h, c.dst, c.dpitch, c.src, c.spitch, c.width, c.height);
}

// After a transform consumed [out0, out0+covered) of a held copy, move the
// parts of the copy it did not cover.
int finish_fused_copy(H *h, const char *out0, size_t covered) {
  HeldCopy c = h->copy;
  h->copy.active = false;
  h->stats.fused_copies++;
  const size_t pre = static_cast<size_t>(out0 - c.dst);
  B2_TRY(issue_copy(h, c.dst, c.src, pre));
  const size_t end = pre + covered;
  if (end < c.bytes)
    B2_TRY(issue_copy(h, c.dst + end, c.src + end, c.bytes - end));
  return B200FFT_SUCCESS;
}

// Launch one pass of plan p. `in`/`out` point at the first transform;
// slabs/slab (complex elements) describe a coalesced middle-axis run.
cudaError_t launch_kernel(H *h, const Plan &p, int dir, const PassArgs &a);

// Kernel arguments of one pass of plan p run by kernel family `family`
// (element units differ between the specialised and generic R2C/C2R kernels).
PassArgs pass_args(const Plan &p, int family, const void *in, void *out, const void *tw,
                   long long slabs, long long slab) {
  PassArgs a{};
  a.in = in;
  a.out = out;
  a.tw = tw;
  a.batch = p.batch;
  a.total = p.batch * slabs;
  if (p.kind == KIND_C2C) {
    a.idist = a.odist = p.dist;
    a.istride = a.ostride = p.stride;
    a.islab = a.oslab = slab;
  } else if (family == 0) { // both sides complex units, contiguous rows
    a.idist = a.odist = p.dist / 2;
    a.istride = a.ostride = 1;
    a.islab = a.oslab = 0;
  } else if (p.kind == KIND_R2C) {
    a.idist = p.dist;
    a.istride = p.stride;
    a.odist = p.dist / 2;
    a.ostride = p.stride;
  } else {
    a.idist = p.dist / 2;
    a.istride = p.stride;
    a.odist = p.dist;
    a.ostride = p.stride;
  }
  return a;
}

long long pass_bytes(const H *h, const Plan &p, long long total) {
  const long long cs = static_cast<long long>(h->csize());
  if (p.kind == KIND_C2C)
    return 2LL * total * p.len * cs;
  return total * (p.len * static_cast<long long>(h->rsize) + (p.len / 2 + 1) * cs);
}

// in_dist >= 0 replaces the input row distance (in the kernel's input units):
// the R2C pass of a fused pad reads the unpadded source rows.
int launch_pass(H *h, const Plan &p, int dir, const void *in, void *out,
                long long slabs, long long slab, bool fused, int stage, long long in_dist = -1) {
  const void *tw = nullptr;
  B2_TRY(get_table(h, p.ch.tlen, &tw));
  PassArgs a = pass_args(p, p.ch.family, in, out, tw, slabs, slab);
  if (in_dist >= 0)
    a.idist = in_dist;
  const long long bytes = pass_bytes(h, p, a.total);
  if (h->recording) { // inside a group: the group launches it later
    RecOp op;
    op.type = RecOp::PASS;
    op.plan = p;
    op.dir = dir;
    op.in = in;
    op.out = out;
    op.tw = tw;
    op.slabs = slabs;
    op.slab = slab;
    h->recs.push_back(op);
    h->stats.bytes_transformed += static_cast<uint64_t>(bytes);
    return B200FFT_SUCCESS;
  }
  h->stats.kernel_launches++;
  h->stats.bytes_transformed += static_cast<uint64_t>(bytes);
  b200fft_launch_record r{};
  r.kind = p.kind;
  r.direction = dir;
  r.stage = stage;
  r.family = p.ch.family;
  r.length = p.len;
  r.fused_copy = fused ? 1 : 0;
  r.transforms = a.total;
  r.slabs = slabs;
  r.bytes = bytes;
  if (h->record_only || a.total == 0) {
    push_log(h, r);
    return B200FFT_SUCCESS;
  }
  ProfileScope ps(h);
  h->last_tma = false;
  const cudaError_t e = launch_kernel(h, p, dir, a);
  if (h->last_tma)
    r.family = 4;
  push_log(h, r);
  ps.done();
  if (e != cudaSuccess)
    return cuda_fail(e, "transform kernel launch");
  return B200FFT_SUCCESS;
}

// The kernel launch of one pass (no bookkeeping).
int device_sms(int dev) {
  static std::atomic<int> n[32] = {}; // per device; every thread stores the same value
  if (dev < 0 || dev >= 32)
    return 148;
  int v = n[dev].load();
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    n[dev].store(v);
  }
  return v;
}

// Tile of a specialised column pass at launch: a pass too small to give every
// SM two full tiles (e.g. a 64^3 grid) takes the half or quarter tile, so more
// CTAs share its latency. Only the Estimate default is adjusted; measured
// plans keep their choice.
int column_tile_for(const H *h, const Plan &p, long long total) {
  int var = p.ch.variant;
  if (h->plan_flag != B200FFT_PLAN_ESTIMATE || !p.ch.col || !is_pow2(p.ch.L) ||
      (var != 0 && var != 5))
    return var;
  const long long want = 2ll * device_sms(h->device);
  const int csz = h->csize();
  if ((total + cfg_static(csz, p.ch.L, true, var).TB - 1) / cfg_static(csz, p.ch.L, true, var).TB >=
      want)
    return var;
  for (int v = 1; v <= 2; ++v)
    if ((total + cfg_static(csz, p.ch.L, true, v).TB - 1) / cfg_static(csz, p.ch.L, true, v).TB >=
        want)
      return v;
  return 2;
}

cudaError_t launch_kernel(H *h, const Plan &p, int dir, const PassArgs &a) {
  const bool f64 = h->prec == B200FFT_F64;
  const bool fwd = dir == B200FFT_FORWARD;
  cudaError_t e;
  if (p.ch.family == 0) {
    if (p.kind == KIND_C2C) {
      int var = column_tile_for(h, p, a.total);
      // FP32 512-point columns whose neighbouring transforms sit side by side
      // on 16-byte aligned rows (the first axis of a grid) take the pair tile
      // by default: 16-byte loads, stores and exchanges (512^3 first-axis
      // pass 0.212 -> 0.195 ms); odd point strides keep the one-transform
      // tile (the pair tile's 8-byte form was slower there, 0.237 vs 0.225 ms,
      // and so was the TMA double-row kernel, 0.235 ms)
      if (var == 5 && h->plan_flag == B200FFT_PLAN_ESTIMATE && !f64 && p.ch.col &&
          p.ch.L == 512 && colpair_vec_ok(a))
        var = kVariantPair;
      if (var == kVariantPair && !f64 && p.ch.col && colpair_length_ok(p.ch.L))
        return launch_colpair_c2c_f32(p.ch.L, fwd, a, h->stream);
      if (var == kVariantTma || var == kVariantTma + 1) {
        if (!f64 && p.ch.col && tma_col_ok(p.ch.L, a)) {
          h->used_tma = true;
          h->last_tma = true;
          return launch_tma_col_c2c_f32(p.ch.L, fwd, var == kVariantTma ? 512 : 1024, a,
                                        h->stream);
        }
        if (!f64 && p.ch.col && tma_mid_ok(p.ch.L, a)) {
          h->used_tma = true;
          h->last_tma = true;
          return launch_tma_mid_c2c_f32(p.ch.L, fwd, var == kVariantTma ? 512 : 1024, a,
                                        h->stream);
        }
        var = default_variant(h->csize(), p.ch.L, p.ch.col, p.stride);
      }
      e = f64 ? launch_static_c2c_f64(p.ch.L, p.ch.col, fwd, var, a, h->stream)
              : launch_static_c2c_f32(p.ch.L, p.ch.col, fwd, var, a, h->stream);
    }
    else if (p.kind == KIND_R2C)
      e = f64 ? launch_static_r2c_f64(p.ch.L, p.ch.variant, a, h->stream)
              : launch_static_r2c_f32(p.ch.L, p.ch.variant, a, h->stream);
    else
      e = f64 ? launch_static_c2r_f64(p.ch.L, p.ch.variant, a, h->stream)
              : launch_static_c2r_f32(p.ch.L, p.ch.variant, a, h->stream);
  } else if (p.ch.family == 2) {
    e = launch_tc_c2c_f32(p.ch.L, p.ch.col, fwd, a, h->stream);
  } else if (p.ch.family == 3) {
    h->used_tc5 = true;
    e = launch_tc5_row256_f32(fwd, a, h->stream);
  } else if (p.ch.family == 5) {
    h->used_tc5 = true;
    e = launch_tc5_col512_f32(fwd, a, h->stream);
  } else {
    GenArgs g = p.ch.gen;
    g.p = a;
    e = launch_generic(f64, p.kind, p.ch.col, fwd, g, h->stream);
  }
  return e;
}

int flush_run(H *h) {
  if (!h->run.active)
    return B200FFT_SUCCESS;
  HeldRun r = h->run;
  h->run.active = false;
  const Plan &p = h->stages[r.stage];
  const char *in = r.out0;
  if (r.fused)
    in = h->copy.src + (r.out0 - h->copy.dst);
  const long long slab = r.lead > 1 ? static_cast<long long>(r.slab_bytes / h->csize()) : 0;
  B2_TRY(launch_pass(h, p, r.dir, in, r.out0, r.count, slab, r.fused, r.stage));
  if (r.fused)
    B2_TRY(finish_fused_copy(h, r.out0, static_cast<size_t>(r.count) * r.slab_bytes));
  return B200FFT_SUCCESS;
}

int flush_all(H *h) {
  B2_TRY(flush_run(h));
  B2_TRY(flush_pad(h));
  return flush_copy(h);
}

bool copy_covers(const H *h, const char *p, size_t n) {
  const HeldCopy &c = h->copy;
  return c.active && p >= c.dst && p + n <= c.dst + c.bytes;
}

int check_handle(H *h) {
  if (h == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft: null handle");
  return B200FFT_SUCCESS;
}

bool is_device_ptr(const void *p) {
  cudaPointerAttributes at{};
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice;
}

// ---- plan cache ("wisdom") and autotuner ------------------------------------
// A wisdom entry records, for one plan geometry on one GPU model, the kernel
// candidate that measured fastest and the planning rigor it was measured at
// (1 Measure, 2 Patient). Planning at any rigor reuses an entry measured at
// that rigor or above; b200fft_export_wisdom / b200fft_import_wisdom save and
// load entries as text lines, like FFTW wisdom (fft_backend_fftw.hpp:666-694).
struct WisdomVal {
  int family = 0, variant = 0, rigor = 0;
  double ms = 0.0;
};
std::mutex g_wis_mu;
std::map<std::string, WisdomVal> g_wisdom;

std::string device_tag(const H *h) {
  if (h->record_only)
    return "record-only";
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) {
    cudaGetLastError();
    return "unknown";
  }
  std::string n = prop.name;
  for (char &c : n)
    if (c == ' ')
      c = '_';
  return n + "_sm" + std::to_string(prop.multiProcessorCount);
}

std::string wisdom_key(const H *h, const Plan &p, long long lead) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s p%d k%d n%d b%lld s%lld d%lld l%lld",
                device_tag(h).c_str(), h->prec, p.kind, p.len, p.batch, p.stride, p.dist,
                lead);
  return buf;
}

size_t plan_region_bytes(const H *h, const Plan &p, long long lead) {
  if (p.kind == KIND_C2C)
    return lead > 1 ? static_cast<size_t>(lead) * p.len * p.batch * h->csize()
                    : c2c_span_bytes(h, p);
  return real_span_bytes(h, p);
}

// Time one candidate: 1 warm-up launch, then the mean of 3, in place on `work`.
int time_candidate(H *h, const Plan &q, long long lead, double *ms) {
  const void *tw = nullptr;
  B2_TRY(get_table(h, q.ch.tlen, &tw));
  const long long slab = lead > 1 ? static_cast<long long>(q.len) * q.batch : 0;
  const PassArgs a = pass_args(q, q.ch.family, h->work, h->work, tw, lead, slab);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = launch_kernel(h, q, B200FFT_FORWARD, a);
  if (e == cudaSuccess)
    e = cudaEventRecord(e0, h->stream);
  for (int i = 0; i < 3 && e == cudaSuccess; ++i)
    e = launch_kernel(h, q, i % 2 ? B200FFT_BACKWARD : B200FFT_FORWARD, a);
  if (e == cudaSuccess)
    e = cudaEventRecord(e1, h->stream);
  if (e == cudaSuccess)
    e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess)
    e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) {
    // a candidate that cannot launch here is skipped, not fatal
    cudaGetLastError();
    *ms = -1.0;
    return B200FFT_SUCCESS;
  }
  *ms = t / 3.0;
  return B200FFT_SUCCESS;
}

// Pick the kernel of plan p by timing candidates (Measure: the default and
// its closest alternatives; Patient: every tile shape and the generic
// kernel), unless wisdom already has an answer of sufficient rigor.
int autotune(H *h, Plan &p) {
  const int rigor = h->plan_flag; // 1 Measure, 2 Patient
  const long long lead = infer_lead(h, p);
  const std::string key = wisdom_key(h, p, lead);
  {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    auto it = g_wisdom.find(key);
    if (it != g_wisdom.end() && it->second.rigor >= rigor) {
      Choice c;
      if (choose_kernel(h->prec, p.kind, p.len, p.batch, p.stride, p.dist,
                        it->second.family == 1, &c, it->second.variant) == B200FFT_SUCCESS) {
        p.ch = c;
        return B200FFT_SUCCESS;
      }
    }
  }
  if (h->record_only || h->work == nullptr)
    return B200FFT_SUCCESS; // nothing to time on: keep the default
  const size_t need = plan_region_bytes(h, p, lead);
  if (h->work_bytes != 0 && need > h->work_bytes)
    return B200FFT_SUCCESS;
  std::vector<std::pair<int, int>> cands; // (family, variant)
  if (p.ch.family == 0) {
    if (p.ch.col) {
      const int meas[] = {0, 3, 5, 8, 10};
      const int pat[] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
      if (rigor >= B200FFT_PLAN_PATIENT)
        for (int v : pat) cands.push_back({0, v});
      else
        for (int v : meas) cands.push_back({0, v});
    } else {
      const int nv = rigor >= B200FFT_PLAN_PATIENT ? 3 : 2;
      for (int v = 0; v < nv; ++v)
        cands.push_back({0, v});
    }
  }
  if (rigor >= B200FFT_PLAN_PATIENT || p.ch.family == 1)
    cands.push_back({1, 0});
  double best = -1.0;
  Choice best_c = p.ch;
  WisdomVal wv;
  for (auto fv : cands) {
    Choice c;
    if (choose_kernel(h->prec, p.kind, p.len, p.batch, p.stride, p.dist, fv.first == 1, &c,
                      fv.second) != B200FFT_SUCCESS)
      continue;
    if (c.family != fv.first)
      continue;
    Plan q = p;
    q.ch = c;
    double ms = -1.0;
    B2_TRY(time_candidate(h, q, lead, &ms));
    if (ms > 0 && (best < 0 || ms < best)) {
      best = ms;
      best_c = c;
      wv.family = c.family;
      wv.variant = c.variant;
      wv.rigor = rigor;
      wv.ms = ms;
    }
  }
  if (best > 0) {
    p.ch = best_c;
    std::lock_guard<std::mutex> lk(g_wis_mu);
    g_wisdom[key] = wv;
  }
  return B200FFT_SUCCESS;
}

int make_plan(H *h, Plan *dst, int kind, int length, size_t batch,
              ptrdiff_t stride, ptrdiff_t dist) {
  if (length < 1)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft: length must be >= 1");
  if (batch < 1 || stride < 1 || dist < 1)
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft: batch, stride and dist must be >= 1");
  if (batch > (1ull << 40) || stride > (1ll << 44) || dist > (1ll << 44))
    return fail(B200FFT_ERR_RANGE, "b200fft: plan arguments exceed the supported range");
  if (kind != KIND_C2C && batch > 1 &&
      dist < 2LL * ((length / 2) * static_cast<long long>(stride) + 1))
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft: in-place R2C/C2R rows overlap: dist must be at least "
                "2*((length/2)*stride+1) reals");
  B2_TRY(flush_all(h));
  Plan p;
  p.kind = kind;
  p.len = length;
  p.batch = static_cast<long long>(batch);
  p.stride = stride;
  p.dist = dist;
  B2_TRY(choose_kernel(h->prec, kind, length, p.batch, stride, dist,
                       h->force_generic, &p.ch, -1, h->split_tc));
  const void *tw = nullptr;
  B2_TRY(get_table(h, p.ch.tlen, &tw));
  p.valid = true;
  *dst = p; // visible to infer_lead while tuning
  // The split-precision kernels are a precision choice, not a tuning
  // candidate: plans that use them are not timed against the plain ones.
  if (h->plan_flag >= B200FFT_PLAN_MEASURE && !h->force_generic && p.ch.family < 2 &&
      std::getenv("B200FFT_VARIANT") == nullptr) {
    B2_TRY(autotune(h, p));
    *dst = p;
  }
  return B200FFT_SUCCESS;
}

int exec_real(H *h, Plan &p, int kind, void *ptr) {
  if (ptr == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft: null data pointer");
  if (!p.valid)
    return fail(B200FFT_ERR_NO_PLAN, kind == KIND_R2C
                                         ? "b200fft: execute_r2c_inplace before create_r2c_inplace_plan"
                                         : "b200fft: execute_c2r_inplace before create_c2r_inplace_plan");
  h->stats.exec_calls++;
  B2_TRY(flush_run(h));
  if (h->pad.active) {
    // A held pad copy whose rows are exactly this R2C plan's rows: the pass
    // reads the unpadded source rows and writes the padded output (every
    // padded row is overwritten whole, pad lanes included).
    const HeldCopy2D c = h->pad;
    const size_t rs = static_cast<size_t>(h->rsize);
    const size_t unit = p.ch.family == 0 ? 2 * rs : rs; // input units of the kernel
    const char *src_end = c.src + c.spitch * (c.height - 1) + c.width;
    const char *dst_end = c.dst + c.dpitch * c.height;
    const bool match = kind == KIND_R2C && c.dst == ptr && p.stride == 1 &&
                       c.width == static_cast<size_t>(p.len) * rs &&
                       c.height == static_cast<size_t>(p.batch) &&
                       c.dpitch == static_cast<size_t>(p.dist) * rs && c.spitch % unit == 0 &&
                       reinterpret_cast<uintptr_t>(c.src) % unit == 0 &&
                       (src_end <= c.dst || dst_end <= c.src);
    if (match) {
      h->pad.active = false;
      h->stats.fused_copies++;
      return launch_pass(h, p, B200FFT_FORWARD, c.src, ptr, 1, 0, true, -1,
                         static_cast<long long>(c.spitch / unit));
    }
    B2_TRY(flush_pad(h));
  }
  char *cp = static_cast<char *>(ptr);
  const size_t span = real_span_bytes(h, p);
  // fold a held copy only into contiguous padded rows (no gaps the pass
  // would skip; a C2R pass leaves each row's two pad reals unspecified, as
  // an in-place C2R does)
  const bool dense = p.stride == 1 && p.dist == 2 * (p.len / 2 + 1);
  bool fused = false;
  if (h->copy.active) {
    if (dense && copy_covers(h, cp, span))
      fused = true;
    else
      B2_TRY(flush_copy(h));
  }
  const void *in = fused ? static_cast<const void *>(h->copy.src + (cp - h->copy.dst)) : ptr;
  const int dir = kind == KIND_R2C ? B200FFT_FORWARD : B200FFT_BACKWARD;
  B2_TRY(launch_pass(h, p, dir, in, ptr, 1, 0, fused, -1));
  if (fused)
    B2_TRY(finish_fused_copy(h, cp, span));
  return B200FFT_SUCCESS;
}

void *record_alloc(size_t bytes) {
  void *p = nullptr;
  if (posix_memalign(&p, 256, bytes ? bytes : 1) != 0)
    return nullptr;
  return p; // pages stay untouched: record-only handles never move data
}

} // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char *b200fft_last_error(void) { return g_err.c_str(); }

int b200fft_version(void) { return 100; }

int b200fft_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int b200fft_create(int precision, int num_stages, int plan_flag, unsigned flags,
                   b200fft_handle *out) {
  if (out == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_create: null output");
  *out = nullptr;
  if (precision != B200FFT_F32 && precision != B200FFT_F64)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_create: precision must be B200FFT_F32 or B200FFT_F64");
  if (num_stages < 0 || num_stages > 64)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_create: num_stages out of range");
  if (plan_flag < B200FFT_PLAN_ESTIMATE || plan_flag > B200FFT_PLAN_PATIENT)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_create: unknown plan flag");
  if (env_flag("B200FFT_RECORD_ONLY"))
    flags |= B200FFT_FLAG_RECORD_ONLY;
  if (env_flag("B200FFT_NO_DEFER"))
    flags |= B200FFT_FLAG_NO_DEFER;
  if (env_flag("B200FFT_GENERIC_ONLY"))
    flags |= B200FFT_FLAG_GENERIC_ONLY;
  if (env_flag("B200FFT_SPLIT_TC"))
    flags |= B200FFT_FLAG_SPLIT_TC;
  static std::once_flag wisdom_once; // B200FFT_WISDOM=path: import once per process
  std::call_once(wisdom_once, [] {
    if (const char *w = std::getenv("B200FFT_WISDOM"))
      if (w[0] != '\0')
        b200fft_import_wisdom(w);
  });
  H *h = new H();
  h->prec = precision;
  h->rsize = precision == B200FFT_F64 ? 8 : 4;
  h->nstages = num_stages;
  h->plan_flag = plan_flag;
  h->flags = flags;
  h->record_only = (flags & B200FFT_FLAG_RECORD_ONLY) != 0;
  h->defer = (flags & B200FFT_FLAG_NO_DEFER) == 0;
  h->force_generic = (flags & B200FFT_FLAG_GENERIC_ONLY) != 0;
  h->split_tc = (flags & B200FFT_FLAG_SPLIT_TC) != 0;
  h->stages.resize(num_stages);
  if (!h->record_only) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      delete h;
      return fail(B200FFT_ERR_NO_DEVICE,
                  "b200fft_create: no CUDA device is visible; the B200 backend has no CPU path");
    }
    cudaGetDevice(&h->device);
    cudaError_t e = cudaStreamCreate(&h->own);
    if (e != cudaSuccess) {
      delete h;
      return cuda_fail(e, "cudaStreamCreate");
    }
    h->stream = h->own;
  }
  *out = h;
  return B200FFT_SUCCESS;
}

int b200fft_destroy(b200fft_handle h) {
  if (h == nullptr)
    return B200FFT_SUCCESS;
  h->recording = false;
  int rc = flush_all(h);
  if (h->group != nullptr) { // leave the group first
    auto &v = h->group->handles;
    v.erase(std::remove(v.begin(), v.end(), h), v.end());
    if (!h->record_only && h->stream)
      cudaStreamSynchronize(h->stream);
    h->group = nullptr;
    h->stream = h->own;
  }
  if (!h->record_only) {
    if (h->stream)
      cudaStreamSynchronize(h->stream);
    resolve_timings(h);
    for (cudaEvent_t e : h->event_pool)
      cudaEventDestroy(e);
    for (auto &kv : h->tables)
      cudaFree(kv.second);
    if (h->own)
      cudaStreamDestroy(h->own);
  }
  delete h;
  return rc;
}

int b200fft_set_stream(b200fft_handle h, void *cuda_stream) {
  B2_TRY(check_handle(h));
  B2_TRY(flush_all(h));
  h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own;
  return B200FFT_SUCCESS;
}

int b200fft_plan_c2c(b200fft_handle h, int stage, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist) {
  B2_TRY(check_handle(h));
  if (stage < 0 || stage >= h->nstages)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_plan_c2c: stage " + std::to_string(stage) +
                                             " outside [0, num_stages)");
  return make_plan(h, &h->stages[stage], KIND_C2C, length, batch, stride, dist);
}

int b200fft_exec_c2c(b200fft_handle h, int stage, int direction, void *data) {
  B2_TRY(check_handle(h));
  if (stage < 0 || stage >= h->nstages)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_exec_c2c: stage out of range");
  if (direction != B200FFT_FORWARD && direction != B200FFT_BACKWARD)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_exec_c2c: bad direction");
  if (data == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_exec_c2c: null data pointer");
  Plan &p = h->stages[stage];
  if (!p.valid)
    return fail(B200FFT_ERR_NO_PLAN, "b200fft_exec_c2c: stage " + std::to_string(stage) +
                                         " has no plan");
  h->stats.exec_calls++;
  char *cp = static_cast<char *>(data);
  HeldRun &r = h->run;
  if (r.active && r.stage == stage && r.dir == direction && r.count < r.lead &&
      cp == r.out0 + static_cast<size_t>(r.count) * r.slab_bytes) {
    r.count++;
    h->stats.coalesced_calls++;
    if (r.count == r.lead)
      return flush_run(h);
    return B200FFT_SUCCESS;
  }
  B2_TRY(flush_run(h));
  B2_TRY(flush_pad(h));
  const long long lead = infer_lead(h, p);
  const size_t slab_bytes = lead > 1 ? static_cast<size_t>(p.len) * p.batch * h->csize()
                                     : c2c_span_bytes(h, p);
  const size_t region = static_cast<size_t>(lead) * slab_bytes;
  // A held copy folds into the pass only when the pass writes every element
  // of its region (no gaps between point rows or transforms): elements a
  // pass skips would otherwise miss their copy.
  const bool dense = lead > 1 || static_cast<size_t>(p.len) * static_cast<size_t>(p.batch) *
                                         h->csize() == slab_bytes;
  bool fused = false;
  if (h->copy.active) {
    if (dense && copy_covers(h, cp, region))
      fused = true;
    else
      B2_TRY(flush_copy(h));
  }
  r.active = true;
  r.stage = stage;
  r.dir = direction;
  r.out0 = cp;
  r.count = 1;
  r.lead = lead;
  r.slab_bytes = slab_bytes;
  r.fused = fused;
  if (lead == 1)
    return flush_run(h);
  return B200FFT_SUCCESS;
}

int b200fft_plan_r2c(b200fft_handle h, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist) {
  B2_TRY(check_handle(h));
  return make_plan(h, &h->r2c, KIND_R2C, length, batch, stride, dist);
}

int b200fft_exec_r2c(b200fft_handle h, void *padded_real) {
  B2_TRY(check_handle(h));
  return exec_real(h, h->r2c, KIND_R2C, padded_real);
}

int b200fft_plan_c2r(b200fft_handle h, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist) {
  B2_TRY(check_handle(h));
  return make_plan(h, &h->c2r, KIND_C2R, length, batch, stride, dist);
}

int b200fft_exec_c2r(b200fft_handle h, void *padded_real) {
  B2_TRY(check_handle(h));
  return exec_real(h, h->c2r, KIND_C2R, padded_real);
}

int b200fft_memcpy(b200fft_handle h, void *dst, const void *src, size_t bytes) {
  B2_TRY(check_handle(h));
  h->stats.memcpy_calls++;
  B2_TRY(flush_all(h));
  if (bytes == 0 || dst == src)
    return B200FFT_SUCCESS;
  if (dst == nullptr || src == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_memcpy: null pointer");
  const char *s = static_cast<const char *>(src);
  char *d = static_cast<char *>(dst);
  const bool hold = h->defer && !overlaps(d, bytes, s, bytes) &&
                    (h->record_only || (is_device_ptr(dst) && is_device_ptr(src)));
  if (hold) {
    h->copy.active = true;
    h->copy.dst = d;
    h->copy.src = s;
    h->copy.bytes = bytes;
    return B200FFT_SUCCESS;
  }
  return issue_copy(h, dst, src, bytes);
}

int b200fft_memcpy2d(b200fft_handle h, void *dst, size_t dpitch, const void *src,
                     size_t spitch, size_t width, size_t height) {
  B2_TRY(check_handle(h));
  h->stats.memcpy_calls++;
  B2_TRY(flush_all(h));
  if (width == 0 || height == 0)
    return B200FFT_SUCCESS;
  if (h->recording) {
    RecOp op;
    op.type = RecOp::COPY2D;
    op.dst = dst;
    op.src = src;
    op.dpitch = dpitch;
    op.spitch = spitch;
    op.width = width;
    op.height = height;
    h->recs.push_back(op);
    return B200FFT_SUCCESS;
  }
  // Device-to-device copies are held: an R2C pass on the same rows takes
  // them over (see exec_real); anything else issues them first.
  if (h->defer && (h->record_only || (is_device_ptr(dst) && is_device_ptr(src)))) {
    h->pad.active = true;
    h->pad.dst = static_cast<char *>(dst);
    h->pad.src = static_cast<const char *>(src);
    h->pad.dpitch = dpitch;
    h->pad.spitch = spitch;
    h->pad.width = width;
    h->pad.height = height;
    return B200FFT_SUCCESS;
  }
  return issue_copy2d(h, dst, dpitch, src, spitch, width, height);
}

int b200fft_flush(b200fft_handle h) {
  B2_TRY(check_handle(h));
  return flush_all(h);
}

int b200fft_sync(b200fft_handle h) {
  B2_TRY(check_handle(h));
  B2_TRY(flush_all(h));
  if (h->record_only || h->recording) // inside a group: b200fft_group_sync waits
    return B200FFT_SUCCESS;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaStreamSynchronize");
  if (h->used_tma) {
    unsigned fault = 0;
    e = tma_take_fault(&fault);
    if (e != cudaSuccess)
      return cuda_fail(e, "TMA column kernel fault word");
    if (fault)
      return fail(B200FFT_ERR_DEVICE_STATUS,
                  "b200fft: a TMA column kernel gave up waiting for its tile copies "
                  "(results of that launch are invalid)");
  }
  if (h->used_tc5) {
    unsigned fault = 0, fault_col = 0;
    e = tc5_take_fault(&fault);
    if (e == cudaSuccess)
      e = tc5col_take_fault(&fault_col);
    if (e != cudaSuccess)
      return cuda_fail(e, "tensor-core fault word");
    fault |= fault_col;
    if (fault)
      return fail(B200FFT_ERR_DEVICE_STATUS,
                  "b200fft: a tensor-core kernel gave up waiting for its products "
                  "(results of that launch are invalid)");
  }
  return B200FFT_SUCCESS;
}

int b200fft_alloc(size_t bytes, void **ptr) {
  if (ptr == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_alloc: null output");
  *ptr = nullptr;
  if (bytes == 0)
    return B200FFT_SUCCESS;
  if (env_flag("B200FFT_RECORD_ONLY")) {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    *ptr = record_alloc(bytes);
    return *ptr ? B200FFT_SUCCESS : fail(B200FFT_ERR_RANGE, "b200fft_alloc: host allocation failed");
  }
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  return B200FFT_SUCCESS;
}

int b200fft_free(void *ptr) {
  if (ptr == nullptr)
    return B200FFT_SUCCESS;
  if (env_flag("B200FFT_RECORD_ONLY")) {
    std::free(ptr);
    return B200FFT_SUCCESS;
  }
  cudaError_t e = cudaFree(ptr);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaFree");
  return B200FFT_SUCCESS;
}

int b200fft_set_profiling(b200fft_handle h, int on) {
  B2_TRY(check_handle(h));
  B2_TRY(flush_all(h));
  h->profiling = on != 0;
  return B200FFT_SUCCESS;
}

int b200fft_set_work_buffer(b200fft_handle h, void *work, size_t bytes) {
  B2_TRY(check_handle(h));
  h->work = work;
  h->work_bytes = bytes;
  return B200FFT_SUCCESS;
}

int b200fft_plan_describe(b200fft_handle h, int kind, int stage, char *buf, size_t buflen) {
  B2_TRY(check_handle(h));
  if (buf == nullptr || buflen == 0)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_plan_describe: null buffer");
  const Plan *p = nullptr;
  if (kind == KIND_C2C) {
    if (stage < 0 || stage >= h->nstages)
      return fail(B200FFT_ERR_INVALID_ARG, "b200fft_plan_describe: stage out of range");
    p = &h->stages[stage];
  } else if (kind == KIND_R2C) {
    p = &h->r2c;
  } else if (kind == KIND_C2R) {
    p = &h->c2r;
  } else {
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_plan_describe: bad kind");
  }
  if (!p->valid)
    return fail(B200FFT_ERR_NO_PLAN, "b200fft_plan_describe: no such plan");
  std::snprintf(buf, buflen, "%s", describe_choice(p->ch, p->kind).c_str());
  return B200FFT_SUCCESS;
}

int b200fft_export_wisdom(const char *path) {
  if (path == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_export_wisdom: null path");
  FILE *f = std::fopen(path, "w");
  if (f == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, std::string("b200fft_export_wisdom: cannot write ") + path);
  std::fprintf(f, "b200fft-wisdom 1\n");
  {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    for (const auto &kv : g_wisdom)
      std::fprintf(f, "%s | %d %d %d %.6f\n", kv.first.c_str(), kv.second.family,
                   kv.second.variant, kv.second.rigor, kv.second.ms);
  }
  std::fclose(f);
  return B200FFT_SUCCESS;
}

int b200fft_import_wisdom(const char *path) {
  if (path == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_import_wisdom: null path");
  FILE *f = std::fopen(path, "r");
  if (f == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, std::string("b200fft_import_wisdom: cannot read ") + path);
  char line[512];
  int n = 0;
  bool header = false;
  while (std::fgets(line, sizeof(line), f)) {
    std::string l(line);
    while (!l.empty() && (l.back() == '\n' || l.back() == '\r'))
      l.pop_back();
    if (!header) {
      header = l == "b200fft-wisdom 1";
      if (!header) {
        std::fclose(f);
        return fail(B200FFT_ERR_INVALID_ARG, "b200fft_import_wisdom: not a wisdom file");
      }
      continue;
    }
    const size_t bar = l.find(" | ");
    if (bar == std::string::npos)
      continue;
    WisdomVal v;
    if (std::sscanf(l.c_str() + bar + 3, "%d %d %d %lf", &v.family, &v.variant, &v.rigor,
                    &v.ms) != 4)
      continue;
    if (v.family < 0 || v.family > 1 || v.variant < 0 || v.variant >= kStaticVariants ||
        v.rigor < 0 || v.rigor > 2)
      continue;
    std::lock_guard<std::mutex> lk(g_wis_mu);
    g_wisdom[l.substr(0, bar)] = v;
    ++n;
  }
  std::fclose(f);
  return n;
}

int b200fft_forget_wisdom(void) {
  std::lock_guard<std::mutex> lk(g_wis_mu);
  g_wisdom.clear();
  return B200FFT_SUCCESS;
}

int b200fft_get_stats(b200fft_handle h, b200fft_stats *out) {
  B2_TRY(check_handle(h));
  if (out == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_get_stats: null output");
  *out = h->stats;
  return B200FFT_SUCCESS;
}

int b200fft_reset_stats(b200fft_handle h) {
  B2_TRY(check_handle(h));
  if (!h->record_only)
    resolve_timings(h);
  h->stats = b200fft_stats{};
  h->log_base += h->log.size();
  h->log.clear();
  return B200FFT_SUCCESS;
}

int b200fft_get_log(b200fft_handle h, b200fft_launch_record *out, int cap,
                    int *count) {
  B2_TRY(check_handle(h));
  if (count == nullptr || (cap > 0 && out == nullptr))
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_get_log: null output");
  B2_TRY(flush_all(h));
  if (!h->record_only)
    resolve_timings(h);
  const int n = std::min<int>(cap, static_cast<int>(h->log.size()));
  const int start = static_cast<int>(h->log.size()) - n;
  for (int i = 0; i < n; ++i)
    out[i] = h->log[start + i];
  *count = n;
  return B200FFT_SUCCESS;
}

int b200fft_describe(int precision, int kind, int length, size_t batch,
                     ptrdiff_t stride, ptrdiff_t dist, char *buf, size_t buflen) {
  if (buf == nullptr || buflen == 0)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_describe: null buffer");
  if (kind < 0 || kind > 2 || length < 1 || batch < 1 || stride < 1 || dist < 1)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_describe: bad arguments");
  Choice ch;
  B2_TRY(choose_kernel(precision, kind, length, static_cast<long long>(batch), stride,
                       dist, false, &ch));
  std::string s = describe_choice(ch, kind);
  std::snprintf(buf, buflen, "%s", s.c_str());
  return B200FFT_SUCCESS;
}

int b200fft_supported(int precision, int kind, int length) {
  if (length < 1 || kind < 0 || kind > 2)
    return 0;
  Choice ch;
  std::string keep = g_err;
  const int rc = choose_kernel(precision, kind, length, 1, 1, kind == KIND_C2C ? length : 2 * (length / 2 + 1), false, &ch);
  g_err = keep;
  return rc == B200FFT_SUCCESS ? 1 : 0;
}

} // extern "C"

// ============================================================================
// Groups: many handles transformed together (independent grids).
// ============================================================================
namespace {

using G = b200fft_group_s;

void group_free_schedule(G *g) {
  if (g->gexec)
    cudaGraphExecDestroy(g->gexec);
  if (g->graph)
    cudaGraphDestroy(g->graph);
  g->gexec = nullptr;
  g->graph = nullptr;
  if (!g->record_only) {
    for (GroupStep &s : g->steps) {
      if (s.d_items)
        cudaFree(s.d_items);
      if (s.d_sitems)
        cudaFree(s.d_sitems);
      if (s.d_tile_start)
        cudaFree(s.d_tile_start);
      if (s.d_tile_map)
        cudaFree(s.d_tile_map);
    }
    if (g->d_queues)
      cudaFree(g->d_queues);
    for (size_t c = 0; c < g->lanes.size(); ++c)
      for (size_t w = 0; w < g->lanes[c].size(); ++w)
        if (!(c == 0 && w == 0) && g->lanes[c][w])
          cudaStreamDestroy(g->lanes[c][w]);
    for (auto &v : g->lane_done)
      for (cudaEvent_t e : v)
        if (e)
          cudaEventDestroy(e);
    for (cudaEvent_t e : g->chain_start)
      if (e)
        cudaEventDestroy(e);
    if (g->fork_ev)
      cudaEventDestroy(g->fork_ev);
  }
  if (!g->record_only) {
    if (g->d_spasses)
      cudaFree(g->d_spasses);
    if (g->d_sorder)
      cudaFree(g->d_sorder);
    if (g->d_sdone)
      cudaFree(g->d_sdone);
  }
  g->sched = false;
  g->spasses.clear();
  g->sorder.clear();
  g->d_spasses = nullptr;
  g->d_sorder = nullptr;
  g->d_sdone = nullptr;
  g->d_sclaim = nullptr;
  g->sbytes = 0;
  g->lanes.clear();
  g->lane_done.clear();
  g->chain_start.clear();
  g->fork_ev = nullptr;
  g->chains = 1;
  g->d_queues = nullptr;
  g->nqueues = 0;
  g->steps.clear();
}

int sm_count_current() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    n = 148;
  }
  return n;
}

// Whether no two members of the group touch the same memory in their
// recorded operations (each member's passes and copies as byte intervals,
// over-approximated per pass by its padded extent). Forms of the schedule
// that run one member's later passes beside another member's earlier ones
// (chains, the dependency-scheduled kernel) need it; the level barriers of
// one chain do not.
bool members_disjoint(const G *g) {
  struct Span {
    uintptr_t lo, hi;
  };
  std::vector<Span> spans; // every member's memory, as disjoint intervals
  for (const H *h : g->handles) {
    std::vector<Span> own;
    const size_t cs = h->csize(), rs = static_cast<size_t>(h->rsize);
    auto add = [&](const void *p, size_t bytes) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(p);
      own.push_back({a, a + bytes});
    };
    for (const RecOp &op : h->recs) {
      if (op.type == RecOp::COPY) {
        add(op.dst, op.bytes);
        add(op.src, op.bytes);
      } else if (op.type == RecOp::COPY2D) {
        add(op.dst, op.dpitch * (op.height - 1) + op.width);
        add(op.src, op.spitch * (op.height - 1) + op.width);
      } else {
        const Plan &p = op.plan;
        size_t bytes;
        if (p.kind == KIND_C2C) {
          const long long span = static_cast<long long>(p.len - 1) * p.stride +
                                 (p.batch - 1) * p.dist + 1;
          bytes = static_cast<size_t>((op.slabs - 1) * op.slab + span) * cs;
        } else { // padded real rows, dist in reals
          bytes = static_cast<size_t>((p.batch - 1) * p.dist +
                                      2ll * (p.len / 2 + 1) * p.stride) * rs;
        }
        add(op.in, bytes);
        add(op.out, bytes);
      }
    }
    // union of this member's intervals (its operations share its buffers)
    std::sort(own.begin(), own.end(), [](const Span &a, const Span &b) { return a.lo < b.lo; });
    const size_t first = spans.size();
    for (const Span &x : own) {
      if (spans.size() > first && x.lo <= spans.back().hi)
        spans.back().hi = std::max(spans.back().hi, x.hi);
      else
        spans.push_back(x);
    }
  }
  // sorted by start, each interval begins at or after the furthest end before
  // it (a member's own intervals are disjoint after the union)
  std::sort(spans.begin(), spans.end(), [](const Span &a, const Span &b) { return a.lo < b.lo; });
  uintptr_t reach = 0;
  for (const Span &x : spans) {
    if (x.lo < reach)
      return false;
    reach = std::max(reach, x.hi);
  }
  return true;
}

// The dependency-scheduled form of a group (fft_sched.cu), chosen with
// B200FFT_GROUP_SCHEDULE=1. It applies when every member is FP32, every
// recorded operation is a pass whose specialised tile the schedule kernel
// carries, and no two members touch the same memory (grids are then
// independent, so only each grid's own passes order one another). Returns
// false (and leaves g untouched) where it does not apply. It is not the
// default: on 256 uneven grids the one persistent launch took 2.6 ms against
// 2.2 ms for the per-level launches of specialised kernels (its tiles run
// under one register budget and one instruction stream for all lengths).
bool sched_build(G *g, int *rc) {
  *rc = B200FFT_SUCCESS;
  if (!env_flag("B200FFT_GROUP_SCHEDULE"))
    return false;
  if (!members_disjoint(g))
    return false; // members share memory: keep the level barriers
  std::vector<SchedPass> passes;
  std::vector<std::pair<long long, int>> keyed; // (order key, pass)
  // a pass is listed `lag` keys after its dependency; lag >= 1 keeps every
  // pass after the pass it waits for
  long long lag = 2;
  if (const char *v = std::getenv("B200FFT_SCHED_LAG"))
    lag = std::max(1ll, std::atoll(v));

  long long bytes = 0;
  for (size_t hi = 0; hi < g->handles.size(); ++hi) {
    H *h = g->handles[hi];
    if (h->prec != B200FFT_F32 || h->recs.empty())
      return false;
    int prev = -1;
    for (size_t k = 0; k < h->recs.size(); ++k) {
      const RecOp &op = h->recs[k];
      if (op.type != RecOp::PASS)
        return false;
      const Plan &p = op.plan;
      Choice sc;
      if (h->force_generic ||
          choose_kernel(h->prec, p.kind, p.len, p.batch, p.stride, p.dist, false, &sc, 0) !=
              B200FFT_SUCCESS ||
          sc.family != 0)
        return false;
      const int spec = sched_spec_index(p.kind, sc.col, op.dir == B200FFT_FORWARD, sc.L);
      if (spec < 0)
        return false;
      SchedPass q{};
      q.a = pass_args(p, 0, op.in, op.out, op.tw, op.slabs, op.slab);
      q.spec = spec;
      const long long tb = sched_tile_transforms(spec);
      const long long nt = (q.a.total + tb - 1) / tb;
      if (nt <= 0 || nt > INT_MAX)
        return false;
      q.ntiles = static_cast<unsigned>(nt);
      q.dep = prev;
      q.need = prev >= 0 ? passes[static_cast<size_t>(prev)].ntiles : 0;
      bytes += pass_bytes(h, p, q.a.total);
      prev = static_cast<int>(passes.size());
      keyed.push_back({static_cast<long long>(hi) + lag * static_cast<long long>(k), prev});
      passes.push_back(q);
    }
  }
  // list order: by key; within a key, later passes (of grids further ahead)
  // first, their dependencies being the oldest
  std::stable_sort(keyed.begin(), keyed.end(), [&](const auto &a, const auto &b) {
    if (a.first != b.first)
      return a.first < b.first;
    return a.second > b.second;
  });
  std::vector<int2> order;
  for (const auto &kp : keyed)
    for (unsigned t = 0; t < passes[static_cast<size_t>(kp.second)].ntiles; ++t)
      order.push_back(make_int2(kp.second, static_cast<int>(t)));
  if (env_flag("B200FFT_SCHED_STALL_TEST")) {
    // test hook: the last dependent pass waits for one tile more than exist,
    // so its waits run out (bounded, 20 ms) and the fault path is taken
    for (size_t i = passes.size(); i-- > 0;)
      if (passes[i].dep >= 0) {
        passes[i].need += 1;
        break;
      }
    g->swait_ns = 20000000ull;
  } else {
    g->swait_ns = 1000000000ull;
  }
  g->spasses = std::move(passes);
  g->sorder = std::move(order);
  g->sbytes = bytes;
  g->sched = true;
  if (g->record_only)
    return true;
  const size_t np = g->spasses.size();
  // counters: np per-pass words, padding to 8 bytes, the claim word, the fault word
  const size_t claim_off = (np * sizeof(unsigned) + 7) & ~size_t(7);
  const size_t cbytes = claim_off + sizeof(unsigned long long) + sizeof(unsigned);
  cudaError_t e = cudaMalloc(&g->d_spasses, np * sizeof(SchedPass));
  if (e == cudaSuccess)
    e = cudaMalloc(&g->d_sorder, g->sorder.size() * sizeof(int2));
  if (e == cudaSuccess)
    e = cudaMalloc(&g->d_sdone, cbytes);
  if (e == cudaSuccess) {
    g->d_sclaim = reinterpret_cast<unsigned long long *>(
        reinterpret_cast<char *>(g->d_sdone) + claim_off);
    g->d_sfault = reinterpret_cast<unsigned *>(g->d_sclaim + 1);
    e = cudaMemset(g->d_sdone, 0, cbytes);
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(g->d_spasses, g->spasses.data(), np * sizeof(SchedPass),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(g->d_sorder, g->sorder.data(), g->sorder.size() * sizeof(int2),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = sched_grid(&g->sgrid);
  if (e != cudaSuccess) {
    *rc = cuda_fail(e, "group schedule upload");
    return true;
  }
  return true;
}

// Build the steps of the schedule from the members' recordings.
int group_build(G *g) {
  group_free_schedule(g);
  {
    int rc = B200FFT_SUCCESS;
    if (sched_build(g, &rc))
      return rc;
  }
  size_t depth = 0;
  for (H *h : g->handles)
    depth = std::max(depth, h->recs.size());
  // chains: members split into groups of about equal work (largest first,
  // each to the chain with the least so far)
  // (default: 3 chains from 48 members on: 256 uneven grids 2.18 -> 2.12 ms,
  // the chains' level tails overlapping; one chain below that)
  int chains = g->handles.size() >= 48 ? 3 : 1;
  if (const char *v = std::getenv("B200FFT_GROUP_CHAINS"))
    chains = std::max(1, std::min(4, std::atoi(v)));
  chains = std::max(1, std::min<int>(chains, static_cast<int>(g->handles.size())));
  if (chains > 1 && !members_disjoint(g))
    chains = 1; // members share memory: one chain, every level a barrier
  std::vector<int> chain_of(g->handles.size(), 0);
  if (chains > 1) {
    std::vector<std::pair<double, size_t>> work;
    for (size_t i = 0; i < g->handles.size(); ++i) {
      double w = 0;
      for (const RecOp &op : g->handles[i]->recs)
        if (op.type == RecOp::PASS)
          w += static_cast<double>(op.plan.batch) * op.plan.len * op.slabs;
      work.push_back({w, i});
    }
    std::sort(work.begin(), work.end(), [](const auto &a, const auto &b) {
      return a.first > b.first || (a.first == b.first && a.second < b.second);
    });
    std::vector<double> load(static_cast<size_t>(chains), 0.0);
    for (const auto &wi : work) {
      const size_t c = static_cast<size_t>(std::min_element(load.begin(), load.end()) - load.begin());
      chain_of[wi.second] = static_cast<int>(c);
      load[c] += wi.first;
    }
  }
  g->chains = chains;
  for (int chain = 0; chain < chains; ++chain)
  for (size_t d = 0; d < depth; ++d) {
    const size_t first_step = g->steps.size();
    std::map<long long, size_t> bucket; // (static, L, f64, kind, col, fwd) -> step index
    for (size_t hix = 0; hix < g->handles.size(); ++hix) {
      H *h = g->handles[hix];
      if (chain_of[hix] != chain || d >= h->recs.size())
        continue;
      const RecOp &op = h->recs[d];
      if (op.type != RecOp::PASS) {
        GroupStep s;
        s.type = op.type == RecOp::COPY ? GroupStep::COPY : GroupStep::COPY2D;
        s.op = op;
        g->steps.push_back(s);
        continue;
      }
      const Plan &p = op.plan;
      const bool f64s = h->prec == B200FFT_F64;
      const bool fwds = op.dir == B200FFT_FORWARD;
      // A pass with a specialised kernel joins the grouped launch of that
      // kernel (same length, layout, kind and direction), full tile.
      Choice sc;
      if (!h->force_generic &&
          choose_kernel(h->prec, p.kind, p.len, p.batch, p.stride, p.dist, false, &sc, 0) ==
              B200FFT_SUCCESS &&
          sc.family == 0) {
        const long long key = (1ll << 40) | (static_cast<long long>(sc.L) << 8) |
                              (f64s ? 1 : 0) | (p.kind << 1) | ((sc.col ? 1 : 0) << 3) |
                              ((fwds ? 1 : 0) << 4);
        auto it = bucket.find(key);
        size_t si;
        if (it == bucket.end()) {
          GroupStep s;
          s.type = GroupStep::STATIC;
          s.f64 = f64s;
          s.kind = p.kind;
          s.col = sc.col;
          s.fwd = fwds;
          s.L = sc.L;
          s.tile_start.push_back(0);
          g->steps.push_back(s);
          si = g->steps.size() - 1;
          bucket[key] = si;
        } else {
          si = it->second;
        }
        GroupStep &s = g->steps[si];
        const PassArgs pa = pass_args(p, 0, op.in, op.out, op.tw, op.slabs, op.slab);
        if (s.sitems.empty()) {
          s.h = h;
          s.plan = p;
          s.dir = op.dir;
          s.pa = pass_args(p, p.ch.family, op.in, op.out, op.tw, op.slabs, op.slab);
        }
        const int tb = static_tile_transforms(h->csize(), sc.L, sc.col);
        s.sitems.push_back(pa);
        s.tile_start.push_back(s.tile_start.back() + (pa.total + tb - 1) / tb);
        s.bytes += pass_bytes(h, p, pa.total);
        continue;
      }
      Choice gc;
      B2_TRY(choose_kernel(h->prec, p.kind, p.len, p.batch, p.stride, p.dist, true, &gc));
      GenArgs ga = gc.gen;
      ga.p = pass_args(p, 1, op.in, op.out, op.tw, op.slabs, op.slab);
      const bool f64 = h->prec == B200FFT_F64;
      const bool fwd = op.dir == B200FFT_FORWARD;
      const int key = (f64 ? 1 : 0) | (p.kind << 1) | ((gc.col ? 1 : 0) << 3) | ((fwd ? 1 : 0) << 4);
      auto it = bucket.find(key);
      size_t si;
      if (it == bucket.end()) {
        GroupStep s;
        s.type = GroupStep::PASSES;
        s.f64 = f64;
        s.kind = p.kind;
        s.col = gc.col;
        s.fwd = fwd;
        s.tile_start.push_back(0);
        g->steps.push_back(s);
        si = g->steps.size() - 1;
        bucket[key] = si;
      } else {
        si = it->second;
      }
      GroupStep &s = g->steps[si];
      const long long tiles = (ga.p.total + ga.TB - 1) / ga.TB;
      s.items.push_back(ga);
      s.tile_start.push_back(s.tile_start.back() + tiles);
      s.smem = std::max(s.smem, generic_smem_bytes(f64, ga.TB, ga.L));
      s.bytes += pass_bytes(h, p, ga.p.total);
    }
    // largest launches first: the level's launches take the chain's lanes
    // round robin, so each lane starts with a long one and the short ones
    // fill in behind
    std::stable_sort(g->steps.begin() + static_cast<std::ptrdiff_t>(first_step), g->steps.end(),
                     [](const GroupStep &a, const GroupStep &b) { return a.bytes > b.bytes; });
    for (size_t i = first_step; i < g->steps.size(); ++i) {
      g->steps[i].level = static_cast<int>(d);
      g->steps[i].chain = chain;
      if (g->steps[i].type == GroupStep::STATIC && g->steps[i].sitems.size() == 1)
        g->steps[i].type = GroupStep::SINGLE;
    }
  }
  // lanes (streams) of each chain: as many as its widest level, at most
  // kGroupStreams over all chains; lane 0 of chain 0 is the group's stream
  if (!g->record_only) {
    std::vector<size_t> widest(static_cast<size_t>(chains), 1);
    size_t run = 0;
    for (size_t i = 0; i < g->steps.size(); ++i) {
      const bool same = i > 0 && g->steps[i].level == g->steps[i - 1].level &&
                        g->steps[i].chain == g->steps[i - 1].chain;
      run = same ? run + 1 : 1;
      size_t &w = widest[static_cast<size_t>(g->steps[i].chain)];
      w = std::max(w, run);
    }
    const size_t per_chain = std::max<size_t>(1, kGroupStreams / static_cast<size_t>(chains));
    cudaError_t e = cudaSuccess;
    if (chains > 1)
      e = cudaEventCreateWithFlags(&g->fork_ev, cudaEventDisableTiming);
    g->lanes.resize(static_cast<size_t>(chains));
    g->lane_done.resize(static_cast<size_t>(chains));
    g->chain_start.assign(static_cast<size_t>(chains), nullptr);
    for (int c = 0; c < chains && e == cudaSuccess; ++c) {
      const size_t nl = std::min(widest[static_cast<size_t>(c)], per_chain);
      e = cudaEventCreateWithFlags(&g->chain_start[static_cast<size_t>(c)], cudaEventDisableTiming);
      for (size_t w = 0; w < nl && e == cudaSuccess; ++w) {
        cudaStream_t st = g->stream;
        if (!(c == 0 && w == 0))
          e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess)
          g->lanes[static_cast<size_t>(c)].push_back(st);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess)
          e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess)
          g->lane_done[static_cast<size_t>(c)].push_back(ev);
      }
    }
    if (e != cudaSuccess)
      return cuda_fail(e, "group streams");
  }
  // device copies of the work lists, one queue counter per grouped launch
  int q = 0;
  for (GroupStep &s : g->steps)
    if (s.type == GroupStep::PASSES)
      s.queue = q++;
  g->nqueues = q;
  if (g->record_only)
    return B200FFT_SUCCESS;
  const int sms = sm_count_current();
  for (GroupStep &s : g->steps) {
    if (s.type != GroupStep::STATIC)
      continue;
    const long long ntiles = s.tile_start.back();
    if (ntiles > INT_MAX)
      return fail(B200FFT_ERR_RANGE, "b200fft: grouped pass has too many tiles");
    std::vector<int2> map(static_cast<size_t>(ntiles));
    for (size_t it = 0; it + 1 < s.tile_start.size(); ++it)
      for (long long t = s.tile_start[it]; t < s.tile_start[it + 1]; ++t)
        map[static_cast<size_t>(t)] =
            make_int2(static_cast<int>(it), static_cast<int>(t - s.tile_start[it]));
    cudaError_t e = cudaMalloc(&s.d_sitems, s.sitems.size() * sizeof(PassArgs));
    if (e == cudaSuccess)
      e = cudaMalloc(&s.d_tile_map, map.size() * sizeof(int2));
    if (e == cudaSuccess)
      e = cudaMemcpy(s.d_sitems, s.sitems.data(), s.sitems.size() * sizeof(PassArgs),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(s.d_tile_map, map.data(), map.size() * sizeof(int2),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
      return cuda_fail(e, "group work list upload");
  }
  for (GroupStep &s : g->steps) {
    if (s.type != GroupStep::PASSES)
      continue;
    cudaError_t e = cudaMalloc(&s.d_items, s.items.size() * sizeof(GenArgs));
    if (e == cudaSuccess)
      e = cudaMalloc(&s.d_tile_start, s.tile_start.size() * sizeof(long long));
    if (e == cudaSuccess)
      e = cudaMemcpy(s.d_items, s.items.data(), s.items.size() * sizeof(GenArgs),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(s.d_tile_start, s.tile_start.data(),
                     s.tile_start.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
      return cuda_fail(e, "group work list upload");
    const int per_sm = std::max<int>(1, std::min<int>(8, static_cast<int>(
                                             (227 * 1024) / (s.smem + 1024))));
    const long long tasks = s.tile_start.back();
    s.grid = static_cast<int>(std::min<long long>(tasks, static_cast<long long>(sms) * per_sm));
  }
  if (q > 0) {
    cudaError_t e = cudaMalloc(&g->d_queues, q * sizeof(unsigned long long));
    if (e != cudaSuccess)
      return cuda_fail(e, "group queue counters");
  }
  return B200FFT_SUCCESS;
}

int group_run(G *g) {
  g->stats.exec_calls++;
  if (g->sched) {
    g->stats.kernel_launches++;
    g->stats.bytes_transformed += static_cast<uint64_t>(g->sbytes);
    if (g->record_only)
      return B200FFT_SUCCESS;
    if (g->d_sdone == nullptr || g->d_spasses == nullptr || g->d_sorder == nullptr)
      return fail(B200FFT_ERR_INVALID_ARG,
                  "b200fft: the group's schedule was not built (b200fft_group_end failed)");
    cudaGetLastError();
    // zero the pass counters and the claim word (not the fault word)
    const size_t claim_end = reinterpret_cast<char *>(g->d_sclaim + 1) -
                             reinterpret_cast<char *>(g->d_sdone);
    cudaError_t e = cudaMemsetAsync(g->d_sdone, 0, claim_end, g->stream);
    if (e != cudaSuccess)
      return cuda_fail(e, "schedule counter reset");
    SchedArgs a{};
    a.passes = g->d_spasses;
    a.items = g->d_sorder;
    a.nitems = static_cast<long long>(g->sorder.size());
    a.done = g->d_sdone;
    a.claim = g->d_sclaim;
    a.fault = g->d_sfault;
    a.wait_ns = g->swait_ns;
    e = launch_sched(a, g->sgrid, g->stream);
    if (e != cudaSuccess)
      return cuda_fail(e, "schedule kernel launch");
    return B200FFT_SUCCESS;
  }
  for (GroupStep &s : g->steps) {
    if (s.type == GroupStep::PASSES || s.type == GroupStep::STATIC ||
        s.type == GroupStep::SINGLE) {
      g->stats.kernel_launches++;
      g->stats.bytes_transformed += static_cast<uint64_t>(s.bytes);
    } else {
      g->stats.copies_issued++;
    }
  }
  if (g->record_only)
    return B200FFT_SUCCESS;
  cudaGetLastError(); // report only errors of the calls below
  if (g->chains > 1) { // fork: every chain starts after the work before the group
    cudaError_t e = cudaEventRecord(g->fork_ev, g->stream);
    for (int c = 1; c < g->chains && e == cudaSuccess; ++c)
      e = cudaStreamWaitEvent(g->lanes[static_cast<size_t>(c)][0], g->fork_ev, 0);
    if (e != cudaSuccess)
      return cuda_fail(e, "group chain fork");
  }
  for (size_t lv = 0; lv < g->steps.size();) {
    size_t lv_end = lv;
    while (lv_end < g->steps.size() && g->steps[lv_end].level == g->steps[lv].level &&
           g->steps[lv_end].chain == g->steps[lv].chain)
      ++lv_end;
    const size_t ch = static_cast<size_t>(g->steps[lv].chain);
    const std::vector<cudaStream_t> &lanes = g->lanes[ch];
    const size_t nstreams = lanes.size();
    cudaStream_t main_st = lanes[0];
    const size_t width = std::min(lv_end - lv, nstreams);
    if (width > 1) { // fork: the level's other lanes start after the previous level
      cudaError_t e = cudaEventRecord(g->chain_start[ch], main_st);
      for (size_t k = 1; k < width && e == cudaSuccess; ++k)
        e = cudaStreamWaitEvent(lanes[k], g->chain_start[ch], 0);
      if (e != cudaSuccess)
        return cuda_fail(e, "group level fork");
    }
    for (size_t i = lv; i < lv_end; ++i) {
      GroupStep &s = g->steps[i];
      cudaStream_t st = lanes[(i - lv) % nstreams];
      cudaError_t e = cudaSuccess;
      const char *what = "grouped pass";
      if (s.type == GroupStep::PASSES) {
        if (s.tile_start.back() == 0)
          continue;
        e = cudaMemsetAsync(g->d_queues + s.queue, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess)
          what = "queue reset";
        else
          e = launch_generic_group(s.f64, s.kind, s.col, s.fwd, s.d_items, s.d_tile_start,
                                   static_cast<int>(s.items.size()), g->d_queues + s.queue,
                                   s.smem, s.grid, st);
      } else if (s.type == GroupStep::STATIC) {
        what = "grouped specialised pass";
        const long long nt = s.tile_start.back();
        if (s.kind == KIND_C2C)
          e = s.f64 ? launch_static_group_c2c_f64(s.L, s.col, s.fwd, s.d_sitems, s.d_tile_map,
                                                  nt, st)
                    : launch_static_group_c2c_f32(s.L, s.col, s.fwd, s.d_sitems, s.d_tile_map,
                                                  nt, st);
        else
          e = s.f64 ? launch_static_group_real_f64(s.L, s.kind == KIND_R2C, s.d_sitems,
                                                   s.d_tile_map, nt, st)
                    : launch_static_group_real_f32(s.L, s.kind == KIND_R2C, s.d_sitems,
                                                   s.d_tile_map, nt, st);
      } else if (s.type == GroupStep::SINGLE) {
        what = "single pass";
        cudaStream_t keep = s.h->stream;
        s.h->stream = st; // the plan's launch goes to this step's stream
        e = launch_kernel(s.h, s.plan, s.dir, s.pa);
        s.h->stream = keep;
      } else if (s.type == GroupStep::COPY) {
        what = "copy";
        e = cudaMemcpyAsync(s.op.dst, s.op.src, s.op.bytes, cudaMemcpyDefault, st);
      } else {
        what = "2D copy";
        e = cudaMemcpy2DAsync(s.op.dst, s.op.dpitch, s.op.src, s.op.spitch, s.op.width,
                              s.op.height, cudaMemcpyDefault, st);
      }
      if (e != cudaSuccess) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "group step %zu (%s, kind %d, %zu items, grid %d, smem %zu)",
                      i, what, s.kind, s.items.size(), s.grid, s.smem);
        return cuda_fail(e, buf);
      }
    }
    if (width > 1) { // join: the chain's next level starts after all of this one
      cudaError_t e = cudaSuccess;
      for (size_t k = 1; k < width && e == cudaSuccess; ++k) {
        e = cudaEventRecord(g->lane_done[ch][k], lanes[k]);
        if (e == cudaSuccess)
          e = cudaStreamWaitEvent(main_st, g->lane_done[ch][k], 0);
      }
      if (e != cudaSuccess)
        return cuda_fail(e, "group level join");
    }
    lv = lv_end;
  }
  if (g->chains > 1) { // join: the group's stream waits for every chain
    cudaError_t e = cudaSuccess;
    for (int c = 1; c < g->chains && e == cudaSuccess; ++c) {
      e = cudaEventRecord(g->lane_done[static_cast<size_t>(c)][0],
                          g->lanes[static_cast<size_t>(c)][0]);
      if (e == cudaSuccess)
        e = cudaStreamWaitEvent(g->stream, g->lane_done[static_cast<size_t>(c)][0], 0);
    }
    if (e != cudaSuccess)
      return cuda_fail(e, "group chain join");
  }
  return B200FFT_SUCCESS;
}

} // namespace

extern "C" {

int b200fft_group_create(b200fft_group *out) {
  if (out == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_create: null output");
  *out = nullptr;
  G *g = new G();
  g->record_only = env_flag("B200FFT_RECORD_ONLY");
  if (!g->record_only) {
    cudaError_t e = cudaStreamCreate(&g->stream);
    if (e != cudaSuccess) {
      delete g;
      return cuda_fail(e, "cudaStreamCreate (group)");
    }
  }
  *out = g;
  return B200FFT_SUCCESS;
}

int b200fft_group_destroy(b200fft_group g) {
  if (g == nullptr)
    return B200FFT_SUCCESS;
  if (!g->record_only && g->stream)
    cudaStreamSynchronize(g->stream);
  for (H *h : g->handles) {
    h->recording = false;
    h->recs.clear();
    h->group = nullptr;
    h->stream = h->own;
  }
  group_free_schedule(g);
  if (!g->record_only && g->stream)
    cudaStreamDestroy(g->stream);
  delete g;
  return B200FFT_SUCCESS;
}

int b200fft_group_add(b200fft_group g, b200fft_handle h) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_add: null group");
  B2_TRY(check_handle(h));
  if (h->group != nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_add: handle already in a group");
  if (h->record_only != g->record_only)
    return fail(B200FFT_ERR_INVALID_ARG,
                "b200fft_group_add: record-only and device handles cannot share a group");
  B2_TRY(flush_all(h));
  if (!h->record_only) {
    // work already queued on the handle's stream finishes before group work
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
      return cuda_fail(e, "cudaStreamSynchronize (group_add)");
    h->stream = g->stream;
  }
  h->group = g;
  g->handles.push_back(h);
  return B200FFT_SUCCESS;
}

int b200fft_group_begin(b200fft_group g) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_begin: null group");
  if (g->recording)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_begin: already recording");
  for (H *h : g->handles) {
    B2_TRY(flush_all(h));
    h->recs.clear();
    h->recording = true;
  }
  g->recording = true;
  return B200FFT_SUCCESS;
}

int b200fft_group_end(b200fft_group g) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_end: null group");
  if (!g->recording)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_end: group_begin was not called");
  int rc = B200FFT_SUCCESS;
  for (H *h : g->handles) {
    const int r = flush_all(h);
    if (rc == B200FFT_SUCCESS)
      rc = r;
    h->recording = false;
  }
  g->recording = false;
  if (rc == B200FFT_SUCCESS)
    rc = group_build(g);
  for (H *h : g->handles)
    h->recs.clear();
  B2_TRY(rc);
  return group_run(g);
}

int b200fft_group_capture(b200fft_group g) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_capture: null group");
  if (g->record_only)
    return B200FFT_SUCCESS;
  if (g->gexec) {
    cudaGraphExecDestroy(g->gexec);
    g->gexec = nullptr;
  }
  if (g->graph) {
    cudaGraphDestroy(g->graph);
    g->graph = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaStreamBeginCapture");
  const b200fft_stats keep = g->stats;
  const int rc = group_run(g);
  g->stats = keep;
  e = cudaStreamEndCapture(g->stream, &g->graph);
  if (rc != B200FFT_SUCCESS)
    return rc;
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&g->gexec, g->graph, 0);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaGraphInstantiate");
  return B200FFT_SUCCESS;
}

int b200fft_group_replay(b200fft_group g) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_replay: null group");
  if (g->gexec == nullptr)
    return group_run(g);
  g->stats.exec_calls++;
  cudaError_t e = cudaGraphLaunch(g->gexec, g->stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaGraphLaunch");
  return B200FFT_SUCCESS;
}

int b200fft_group_sync(b200fft_group g) {
  if (g == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_sync: null group");
  if (g->record_only)
    return B200FFT_SUCCESS;
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaStreamSynchronize (group)");
  if (g->sched && g->d_sfault) {
    unsigned fault = 0;
    e = cudaMemcpy(&fault, g->d_sfault, sizeof(fault), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && fault)
      e = cudaMemset(g->d_sfault, 0, sizeof(unsigned));
    if (e != cudaSuccess)
      return cuda_fail(e, "schedule fault word");
    if (fault)
      return fail(B200FFT_ERR_DEVICE_STATUS,
                  "b200fft: the group schedule kernel gave up waiting for a pass "
                  "(results of that run are invalid)");
  }
  return B200FFT_SUCCESS;
}

int b200fft_group_stats(b200fft_group g, b200fft_stats *out) {
  if (g == nullptr || out == nullptr)
    return fail(B200FFT_ERR_INVALID_ARG, "b200fft_group_stats: null argument");
  *out = g->stats;
  size_t passes = g->sched ? g->spasses.size() : 0;
  for (const GroupStep &s : g->steps)
    passes += s.items.size() + s.sitems.size();
  out->exec_calls = g->stats.exec_calls;
  out->coalesced_calls = passes; // passes in the current schedule
  return B200FFT_SUCCESS;
}

} // extern "C"
