// Specialised C2C kernels, FP64 (column and row layouts, both directions).
#include "fs_launch.cuh"

namespace b200fft {
cudaError_t launch_static_c2c_f64(int L, bool col, bool fwd, int var, const PassArgs &a,
                                  cudaStream_t st) {
  if (col)
    return fwd ? launch_static_switch<double, true, true, KIND_C2C>(L, var, a, st)
               : launch_static_switch<double, true, false, KIND_C2C>(L, var, a, st);
  return fwd ? launch_static_switch<double, false, true, KIND_C2C>(L, var, a, st)
             : launch_static_switch<double, false, false, KIND_C2C>(L, var, a, st);
}
cudaError_t launch_static_group_c2c_f64(int L, bool col, bool fwd, const PassArgs *items,
                                        const int2 *tile_map, long long ntiles,
                                        cudaStream_t st) {
  if (col)
    return fwd ? launch_static_group_switch<double, true, true, KIND_C2C>(L, items, tile_map, ntiles, st)
               : launch_static_group_switch<double, true, false, KIND_C2C>(L, items, tile_map, ntiles, st);
  return fwd ? launch_static_group_switch<double, false, true, KIND_C2C>(L, items, tile_map, ntiles, st)
             : launch_static_group_switch<double, false, false, KIND_C2C>(L, items, tile_map, ntiles, st);
}
} // namespace b200fft
