// Host+device shared definitions of the B200 transform engine: launch
// arguments, kernel configuration rules and the radix schedule.
//
// A "pass" is one batched 1D transform along one axis of a ParaFaFT stage
// buffer. Transform b of a pass starts at element
//     (b / batch) * slab + (b % batch) * dist
// and its points sit `stride` elements apart. `batch`, `dist` and `stride` are
// the plan arguments of Backend::create_stage_plan
// (backend/fft_backend.hpp:83-93); `slab` is the pointer step between the
// consecutive execute_stage calls that ParaFaFT issues for a middle axis
// (parafaft_c2c.hpp:875-896, parafaft_r2c.hpp:1224-1244), which one pass
// covers at once.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace b200fft {

enum : int { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

// Launch arguments shared by all transform kernels. Input and output sides
// carry their own element units: complex elements for C2C; for R2C the input
// side is in reals and the output side in complex elements; for C2R the
// reverse. The specialised R2C/C2R kernels take both sides in complex units.
struct PassArgs {
  const void *in;
  void *out;
  const void *tw;     // twiddle table exp(-2*pi*i*m/tlen), m in [0, tlen)
  long long total;    // transforms in the launch (batch * slabs)
  long long batch;    // transforms per slab
  long long idist, istride, islab;
  long long odist, ostride, oslab;
};

// Division by a runtime constant d < 2^31 for dividends n < 2^31:
//   q = (n * m) >> (32 + s)  with  m = ceil(2^(31 + l) / d),  l = ceil(log2 d),
// s = l - 1 (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994). d == 1 is encoded as m == 0.
struct FastDiv {
  uint32_t m;
  uint32_t s;
  uint32_t d;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{0u, 0u, d};
  if (d <= 1)
    return f;
  uint32_t l = 0;
  while ((1ull << l) < d)
    ++l;
  const unsigned long long num = (1ull << (31 + l)) + d - 1;
  f.m = static_cast<uint32_t>(num / d);
  f.s = l - 1;
  return f;
}

// Runtime-generic kernel limits.
constexpr int kGenMaxStages = 24;
constexpr int kGenMaxPrime = 61; // largest prime radix done by direct DFT
constexpr int kGenThreads = 256;
constexpr int kGenMaxTB = 64; // transforms per generic tile at most
// static shared memory of a generic tile: input and output offsets per transform
constexpr int kGenStaticSmem = 2 * kGenMaxTB * 8;

struct GenArgs {
  PassArgs p;
  int L;       // complex points per transform handled by the stage loop
  int nreal;   // real length for R2C/C2R (0 for C2C)
  int lout;    // outputs per transform written by the store loop
  int nst;     // number of radix stages
  int TB;      // transforms per CTA (power of two)
  int logTB;
  int tscale;  // table index = exponent * tscale
  int odd;     // R2C/C2R of odd real length (full-length complex transform)
  int rad[kGenMaxStages];
  int nsv[kGenMaxStages];
  FastDiv ns[kGenMaxStages];  // divide by Ns (product of earlier radices)
  FastDiv bq[kGenMaxStages];  // divide by L / radix
  FastDiv Ldiv;               // divide by L
  FastDiv Loutdiv;            // divide by lout
};

// ---- compile-time radix schedule for the specialised kernels ------------
// Stockham stage s with radix R reads points j + r*L/R and writes
// (j/Ns)*Ns*R + j%Ns + r*Ns, Ns = product of the radices before s, so the last
// stage writes natural order directly.
// Powers of two whose threads hold at least 16 points (rmax = 16 or 32) take
// the fewest stages of radices up to rmax, as even as possible, larger first
// (1024 = 32x32 or 16x8x8, 512 = 32x16, 256 = 16x16): every stage saved is a
// shared-memory exchange saved. Otherwise the radix order is 8s, then one 4
// or 2, then 5s, then 3s. Rows of other lengths given prow > 0 (the thread
// count mixed_row_threads chose for them) take the even schedule below.
// Returns the stage count; `rest` is what no radix divides (1 for a
// supported length).
constexpr int even_row_schedule(int L, int P, int (&rad)[24]);
constexpr int static_schedule(int L, int rmax, int prow, int (&rad)[24], int &rest) {
  int k = 0;
  if (prow > 0 && (L & (L - 1)) != 0) {
    const int n = even_row_schedule(L, prow, rad);
    if (n > 0) {
      rest = 1;
      return n;
    }
  }
  if (rmax > 8 && L >= 16 && (L & (L - 1)) == 0) {
    int lg = 0, q = 0;
    while ((1 << lg) < L)
      ++lg;
    while ((1 << q) < rmax)
      ++q;
    const int n = (lg + q - 1) / q;
    for (int i = 0; i < n; ++i)
      rad[k++] = 1 << (lg / n + (i < lg % n ? 1 : 0));
    rest = 1;
    return k;
  }
  int m = L;
  while (m % 8 == 0 && m > 1) {
    rad[k++] = 8;
    m /= 8;
  }
  if (m % 4 == 0) {
    rad[k++] = 4;
    m /= 4;
  }
  if (m % 2 == 0) {
    rad[k++] = 2;
    m /= 2;
  }
  while (m % 5 == 0) {
    rad[k++] = 5;
    m /= 5;
  }
  while (m % 3 == 0) {
    rad[k++] = 3;
    m /= 3;
  }
  rest = m;
  return k;
}

// A row of mixed length L = 2^a 3^b 5^c over P = 2^p threads splits evenly at
// every stage when each radix R leaves L/R a multiple of P, i.e. its
// power-of-two radices are at most 2^(a-p) (and 8). That schedule: as few
// power-of-two radices as that allows, as even as possible, larger first,
// then 5s, then 3s. Every stage then fills all P threads, and R2C/C2R rows
// pair their Hermitian halves with warp shuffles (P <= 32). Returns its stage
// count, or 0 when there is none.
constexpr int even_row_schedule(int L, int P, int (&rad)[24]) {
  int a = 0, m = L, p = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++a;
  }
  while ((1 << p) < P)
    ++p;
  const int q = (a - p) < 3 ? (a - p) : 3;
  if (q < 1 || (L % P) != 0)
    return 0;
  int k = 0;
  const int n = (a + q - 1) / q;
  for (int i = 0; i < n; ++i)
    rad[k++] = 1 << (a / n + (i < a % n ? 1 : 0));
  while (m % 5 == 0) {
    rad[k++] = 5;
    m /= 5;
  }
  while (m % 3 == 0) {
    rad[k++] = 3;
    m /= 3;
  }
  return m == 1 ? k : 0;
}

// Threads per row of a mixed-length row kernel with an even schedule: the
// largest power of two 4 <= P <= 32 whose even schedule has at most three
// stages and at most 24 (8-byte elements) / 12 (16-byte elements, whose
// registers fill twice as fast) points per thread; 0: none, the kernel then
// takes P = floor_pow2(L/8) and the default schedule. Two threads per row
// spread a warp's loads over 16 rows, which cost more than the idle lanes it
// saves (40-point rows: 48/52 -> 57/60 us).
constexpr int mixed_row_threads(int L, int esize) {
  int best = 0;
  for (int P = 4; P <= 32; P *= 2) {
    int rad[24] = {};
    const int n = even_row_schedule(L, P, rad);
    if (n > 0 && n <= 3 && L / P <= (esize == 8 ? 24 : 12))
      best = P;
  }
  return best;
}

// The prow argument of static_schedule for a row kernel of P threads per
// transform: P when that is the even-schedule thread count, else 0.
constexpr int even_row_threads(int L, int esize, int P) {
  return ((L & (L - 1)) != 0 && mixed_row_threads(L, esize) == P) ? P : 0;
}

// Largest radix of a specialised kernel whose threads hold E = L*TB/NT points:
// the largest power of two <= E between 8 and 32 (16 for 16-byte elements,
// whose 32-point butterfly would not fit the registers).
constexpr int radix_cap(int esize, int L, int TB, int NT) {
  const int e = (L * TB) / NT;
  const int cap = esize == 8 ? 32 : 16;
  int r = 8;
  while (2 * r <= e && 2 * r <= cap)
    r *= 2;
  return r;
}

template <int L, int RMAX = 8, int PROW = 0> struct SchedS {
  int nst = 0;
  int rad[24] = {};
  int ns[24] = {};
  int rest = 1;
  constexpr SchedS() {
    nst = static_schedule(L, RMAX, PROW, rad, rest);
    int p = 1;
    for (int i = 0; i < nst; ++i) {
      ns[i] = p;
      p *= rad[i];
    }
  }
};

constexpr int ce_min(int a, int b) { return a < b ? a : b; }
constexpr int ce_max(int a, int b) { return a > b ? a : b; }

// ---- shared-memory layout of row tiles -----------------------------------
// A row tile keeps point n of its transform tb at tb*lp + n + (n >> sh): a pad
// element every 2^sh points and a row pitch lp. One element in 16 (8-byte) or
// 8 (16-byte) with lp = L + L/16 suits power-of-two rows; other lengths pick
// (sh, lp) here by scoring every candidate (sh in {2, 3, 4, 5, none}, lp from
// the smallest pitch up by 15) on the exchange accesses of warp 0: the
// Stockham writes and reads between stages and, for R2C rows, the Hermitian
// pair reads. 8-byte elements fall on 16 bank pairs, 16-byte ones on 8 bank
// quads; an access costs the largest number of lanes on one of them (the
// shared-memory wavefronts it takes).
struct RowPad {
  int sh, lp;
};

template <class Sch>
constexpr long long row_pad_cost(const Sch &S, int L, int P, int esize, bool post, int sh,
                                 int lp) {
  const int nb = 128 / esize;
  long long cost = 0;
  int cnt[16] = {};
  for (int s = 0; s < S.nst; ++s) {
    const int R = S.rad[s], Ns = S.ns[s], B = L / R;
    const bool last = s == S.nst - 1;
    for (int phase = 0; phase < 2; ++phase) { // writes of stage s, reads of s+1
      if ((phase == 0 && last && !post) || (phase == 1 && last))
        continue;
      const int Rx = phase == 0 ? R : S.rad[s + 1];
      const int Bx = L / Rx;
      const int Kx = (Bx + P - 1) / P;
      for (int i = 0; i < Kx; ++i)
        for (int r = 0; r < Rx; ++r) {
          for (int b = 0; b < nb; ++b)
            cnt[b] = 0;
          for (int l = 0; l < 32; ++l) {
            const int g = P <= 32 ? l % P : l, tb = P <= 32 ? l / P : 0;
            const int j = g + P * i;
            if (j >= Bx)
              continue;
            const int n = phase == 1 ? j + r * Bx
                          : last     ? j + r * B
                                     : (j / Ns) * Ns * R + j % Ns + r * Ns;
            ++cnt[(tb * lp + n + (n >> sh)) % nb];
          }
          int mx = 0;
          for (int b = 0; b < nb; ++b)
            mx = cnt[b] > mx ? cnt[b] : mx;
          cost += mx;
        }
    }
  }
  if (post) { // R2C: X[k] reads Z[k] and Z[L-k] (k = 0..L, 0 for L)
    const int KO = (L + 1 + P - 1) / P;
    for (int i = 0; i < KO; ++i)
      for (int h = 0; h < 2; ++h) {
        for (int b = 0; b < nb; ++b)
          cnt[b] = 0;
        for (int l = 0; l < 32; ++l) {
          const int g = P <= 32 ? l % P : l, tb = P <= 32 ? l / P : 0;
          const int k = g + P * i;
          if (k > L)
            continue;
          const int n = h == 0 ? (k == L ? 0 : k) : (k == 0 ? 0 : L - k);
          ++cnt[(tb * lp + n + (n >> sh)) % nb];
        }
        int mx = 0;
        for (int b = 0; b < nb; ++b)
          mx = cnt[b] > mx ? cnt[b] : mx;
        cost += mx;
      }
  }
  return cost;
}

// The layout of a row tile of TB transforms (the cheapest candidate whose tile
// stays within 48 KiB or within the default layout's size; ties keep the
// default, then the smaller pitch).
template <class Sch>
constexpr RowPad choose_row_pad(const Sch &S, int L, int P, int TB, int esize, bool post,
                                bool search) {
  const int sh0 = esize == 8 ? 4 : 3;
  RowPad best{sh0, L + (L >> sh0)};
  if (!search)
    return best;
  const long long budget = ce_max(48 * 1024, TB * best.lp * esize);
  long long bc = row_pad_cost(S, L, P, esize, post, best.sh, best.lp);
  const int shs[5] = {2, 3, 4, 5, 30};
  for (int a = 0; a < 5; ++a) {
    const int sh = shs[a];
    const int base = (L - 1) + ((L - 1) >> sh) + 1;
    for (int q = 0; q < 16; ++q) {
      const int lp = base + q;
      if (static_cast<long long>(TB) * lp * esize > budget)
        break;
      const long long c = row_pad_cost(S, L, P, esize, post, sh, lp);
      if (c < bc) {
        bc = c;
        best = RowPad{sh, lp};
      }
    }
  }
  return best;
}

// Configuration of a specialised kernel: NT threads, TB transforms per CTA,
// P = NT/TB threads per transform, E points per thread.
//  * column layout (points strided, neighbouring transforms adjacent in
//    memory): a CTA owns TB adjacent transforms so every point row it loads is
//    a contiguous TB-element segment; target tile 8192 (f32) / 4096 (f64)
//    points, at most 32 / 16 points per thread.
//  * row layout (points contiguous): P threads per transform read contiguous
//    runs; E between 8 and 32 (f32) / 16 (f64).
struct CfgS {
  int NT, TB, P, E;
};


// `variant` selects the tile shape among the candidates the planner (and its
// autotuner) choose from:
//   column layout: 0 = full tile, 1 = half, 2 = quarter (more CTAs per SM,
//                  fewer registers per thread);
//   row layout:    0 = default points per thread, 1 = twice, 2 = half.
//   3 = wide column tile: 512 threads and twice the full tile, so every
//       point row is read as one longer contiguous segment;
//   4 = staged column pass: persistent CTAs of 512 threads, full tile,
//       cp.async double buffering (one CTA per SM);
//   5 = full column tile on 512 threads (half the points per thread);
//   6 = pipelined column pass: persistent CTAs of 256 threads on half tiles,
//       the next tile's points loaded into a second register set while the
//       current one is transformed (two CTAs per SM).
//   7 = wide column tile on 1024 threads (twice the full tile, half the
//       points per thread): wide row segments with 32 warps per SM.
//   8 = TMA-fed column pass (FP32, 256/512/1024 points, 16-byte aligned
//       rows): persistent CTAs of 512 threads stream 64 KiB tiles through a
//       ring of three shared-memory buffers filled by bulk tensor copies;
//   9 = the same on 1024 threads per CTA.
//  10 = pair-column tile (FP32, 256/512/1024 points): 512 (1024) threads, two
//       neighbouring transforms per thread, 16-byte shared-memory exchanges
//       and twiddles shared by the pair (fft_colpair.cuh).
// Where a TMA or pair variant does not apply, the plan's default tile runs
// instead.
constexpr int kStaticVariants = 11;
constexpr int kVariantTma = 8;
constexpr int kVariantPair = 10;
constexpr int kVariantStaged = 4;
constexpr int kVariantPipelined = 6;

constexpr bool is_pow2(long long x) { return x > 0 && (x & (x - 1)) == 0; }
constexpr int floor_pow2(int x) {
  int p = 1;
  while (p * 2 <= x)
    p *= 2;
  return p;
}

constexpr CfgS cfg_static(int esize, int L, bool col, int variant = 0) {
  if (!is_pow2(L)) {
    // Mixed-radix lengths (factors 8, 4, 2, 5, 3): power-of-two tiles and
    // thread counts per transform; columns also take the half tile (variant
    // 1: 10-15 points per thread, more CTAs per SM).
    const int NT = 256;
    const int base = esize == 8 ? 8192 : 4096;
    if (col) {
      const int tile = base >> (variant == 1 ? 1 : 0);
      const int TB = ce_min(NT, floor_pow2(ce_max(1, tile / L)));
      return CfgS{NT, TB, NT / TB, (TB * L + NT - 1) / NT};
    }
    const int Pe = mixed_row_threads(L, esize);
    const int P = Pe > 0 ? Pe : ce_min(NT, floor_pow2(ce_max(1, L / 8)));
    return CfgS{NT, NT / P, P, (L + P - 1) / P};
  }
  if (col && variant == 10 && esize == 8 && (L == 256 || L == 512 || L == 1024)) {
    // pair-column tile: TB/2 transform pairs, 8 points of each per thread
    const int TB = L == 256 ? 32 : 16;
    const int nt = L == 1024 ? 1024 : 512;
    return CfgS{nt, TB, nt / (TB / 2), L / (nt / (TB / 2))};
  }
  if (variant == 10)
    variant = 5; // the pair tile's shape where it does not apply
  const int NT = (col && (variant == 7 || variant == 9)) ? 1024
                 : (col && ((variant >= 3 && variant <= 5) || variant == 8)) ? 512 : 256;
  const int base = esize == 8 ? 8192 : 4096;
  const int target = col ? ((variant == 3 || variant == 7) ? 2 * base
                                         : (variant == 4 || variant == 5 || variant >= 8)
                                               ? base
                                               : variant == 6 ? base / 2 : (base >> variant))
                         : base;
  const int emax = esize == 8 ? 32 : 16;
  if (col) {
    int TB = ce_min(NT, ce_max(1, target / L));
    int P = NT / TB;
    int E = (TB * L) / NT;
    if (E < 1)
      E = 1;
    return CfgS{NT, TB, P, E};
  }
  int E = L / 32;
  if (E < 8)
    E = ce_min(8, L);
  if (variant == 1)
    E *= 2;
  else if (variant == 2 && E > 8)
    E /= 2;
  if (E > emax)
    E = emax;
  if (E > L)
    E = L;
  int P = L / E;
  if (P > NT)
    P = NT;
  int TB = NT / P;
  return CfgS{NT, TB, P, E};
}

// Lengths with a specialised kernel (complex points of the stage loop):
// powers of two up to 4096, and the mixed-radix lengths below (the sides of
// common non-power-of-two grids and their R2C halves).
constexpr int kStaticMaxL = 4096;
constexpr bool static_pow2_ok(int L) { return L >= 2 && L <= kStaticMaxL && is_pow2(L); }
constexpr bool static_mixed_ok(int L) {
  return L == 24 || L == 30 || L == 40 || L == 48 || L == 60 || L == 80 || L == 96 ||
         L == 120 || L == 160 || L == 192 || L == 384 || L == 768;
}
constexpr bool static_length_ok(int L) { return static_pow2_ok(L) || static_mixed_ok(L); }

} // namespace b200fft
