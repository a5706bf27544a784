// Host-side launchers of the transform kernels (defined in fs_*.cu / fg.cu).
#pragma once

#include <cuda_runtime.h>

#include "fft_common.hpp"

namespace b200fft {

// Family S: specialised kernels for power-of-two stage lengths L.
// C2C: col selects the column thread mapping (strided points).
cudaError_t launch_static_c2c_f32(int L, bool col, bool fwd, int var, const PassArgs &a,
                                  cudaStream_t st);
cudaError_t launch_static_c2c_f64(int L, bool col, bool fwd, int var, const PassArgs &a,
                                  cudaStream_t st);
// R2C (forward) / C2R (backward) of real length 2L, contiguous padded rows;
// both sides of `a` in complex units.
cudaError_t launch_static_r2c_f32(int L, int var, const PassArgs &a, cudaStream_t st);
cudaError_t launch_static_c2r_f32(int L, int var, const PassArgs &a, cudaStream_t st);
cudaError_t launch_static_r2c_f64(int L, int var, const PassArgs &a, cudaStream_t st);
cudaError_t launch_static_c2r_f64(int L, int var, const PassArgs &a, cudaStream_t st);

// Grouped Family S passes (full tile): items are the passes' kernel arguments
// (device array); tile_map[t] = (item, tile within the item) for each of the
// ntiles tiles of static_tile_transforms(...) transforms (device array).
cudaError_t launch_static_group_c2c_f32(int L, bool col, bool fwd, const PassArgs *items,
                                        const int2 *tile_map, long long ntiles,
                                        cudaStream_t st);
cudaError_t launch_static_group_c2c_f64(int L, bool col, bool fwd, const PassArgs *items,
                                        const int2 *tile_map, long long ntiles,
                                        cudaStream_t st);
cudaError_t launch_static_group_real_f32(int L, bool r2c, const PassArgs *items,
                                         const int2 *tile_map, long long ntiles,
                                         cudaStream_t st);
cudaError_t launch_static_group_real_f64(int L, bool r2c, const PassArgs *items,
                                         const int2 *tile_map, long long ntiles,
                                         cudaStream_t st);
inline int static_tile_transforms(int esize_complex, int L, bool col) {
  return cfg_static(esize_complex, L, col, 0).TB;
}

// Family T: split-precision tensor-core C2C (FP32 data; lengths 256, 512,
// 1024; row or column tiles).
cudaError_t launch_tc_c2c_f32(int L, bool col, bool fwd, const PassArgs &a, cudaStream_t st);
constexpr bool tc_length_ok(int L) { return L == 256 || L == 512 || L == 1024; }
// The same on the fifth-generation tensor cores (tcgen05, TMEM accumulators):
// FP32 C2C rows of length 256.
cudaError_t launch_tc5_row256_f32(bool fwd, const PassArgs &a, cudaStream_t st);
// FP32 C2C columns of length 512 on tcgen05 (fft_tc5col.cu).
cudaError_t launch_tc5_col512_f32(bool fwd, const PassArgs &a, cudaStream_t st);
// The tcgen05 kernels' device fault words (a bounded wait that ran out),
// returned and cleared; call after the launches' stream is synchronised.
cudaError_t tc5_take_fault(unsigned *fault);
cudaError_t tc5col_take_fault(unsigned *fault);
// TMA-fed FP32 column C2C passes (fft_tma.cu): eligibility (lengths 256, 512,
// 1024; contiguous transforms; 16-byte aligned base, stride and slab
// stride), the launch (nt = 512 or 1024 threads per CTA) and the fault word.
bool tma_col_ok(int L, const PassArgs &a);
cudaError_t launch_tma_col_c2c_f32(int L, bool fwd, int nt, const PassArgs &a, cudaStream_t st);
// the same for odd point strides (double-row map; FP32 256/512 points)
bool tma_mid_ok(int L, const PassArgs &a);
cudaError_t launch_tma_mid_c2c_f32(int L, bool fwd, int nt, const PassArgs &a, cudaStream_t st);
cudaError_t tma_take_fault(unsigned *fault);

// Pair-column C2C kernels (fs_colpair.cu, tile variant kVariantPair): FP32
// columns of 256, 512 or 1024 points, two neighbouring transforms per thread.
bool colpair_length_ok(int L);
// Whether the 16-byte global form applies to pass `a` (complex elements):
// unit transform distance, even point and slab strides, an even batch (no
// pair spans two slabs), 16-byte aligned bases.
bool colpair_vec_ok(const PassArgs &a);
cudaError_t launch_colpair_c2c_f32(int L, bool fwd, const PassArgs &a, cudaStream_t st);

// Family G: runtime-generic kernels.
cudaError_t launch_generic(bool f64, int kind, bool col, bool fwd,
                           const GenArgs &g, cudaStream_t st);
size_t generic_smem_bytes(bool f64, int TB, int L);
// Persistent grouped generic pass over device arrays of items (device
// pointers): CTAs take tiles from *queue (zeroed before the launch).
cudaError_t launch_generic_group(bool f64, int kind, bool col, bool fwd, const GenArgs *items,
                                 const long long *tile_start, int nitems,
                                 unsigned long long *queue, size_t smem, int grid,
                                 cudaStream_t st);
constexpr size_t kGenericSmemLimit = 200 * 1024;

// Dependency-scheduled persistent pass kernel (fft_sched.cu): the passes of
// a group of independent grids in one launch. Pass `dep` (whole pass) must be
// done before any tile of this pass starts; `spec` picks the specialised tile
// code (sched_spec_index).
constexpr int kSchedThreads = 256;
struct SchedPass {
  PassArgs a;
  int spec;      // specialised tile code of the pass
  int dep;       // pass this one waits for (-1: none)
  unsigned need; // tiles of `dep` (all of them)
  unsigned ntiles;
};
struct SchedArgs {
  const SchedPass *passes;
  const int2 *items;         // (pass, tile) in claim order
  long long nitems;
  unsigned *done;            // finished tiles per pass, zeroed before each run
  unsigned long long *claim; // next item, zeroed before each run
  unsigned *fault;           // set when a dependency wait ran out of time
  unsigned long long wait_ns; // bound of one wait
};
// Index of the specialised tile for (kind, layout, direction, length), or -1
// when the schedule kernel does not carry it; transforms per tile of a spec.
int sched_spec_index(int kind, bool col, bool fwd, int L);
int sched_tile_transforms(int spec);
// CTAs of a persistent launch on the current device (all resident at once).
cudaError_t sched_grid(int *grid);
cudaError_t launch_sched(const SchedArgs &s, int grid, cudaStream_t st);

// Entries of the twiddle table of top length n: a pyramid T_n, T_{n/2}, ...,
// T_1 for powers of two (2n - 1 entries), else T_n alone.
int twiddle_table_entries(int n);
// FP64-computed twiddle table of top length n (t64 and/or t32 may be null).
cudaError_t launch_twiddle_table(double2 *t64, float2 *t32, int n,
                                 cudaStream_t st);

} // namespace b200fft
