// Specialised R2C (forward) and C2R (backward) row kernels, FP32.
#include "fs_launch.cuh"

namespace b200fft {
cudaError_t launch_static_r2c_f32(int L, int var, const PassArgs &a, cudaStream_t st) {
  return launch_static_switch<float, false, true, KIND_R2C>(L, var, a, st);
}
cudaError_t launch_static_c2r_f32(int L, int var, const PassArgs &a, cudaStream_t st) {
  return launch_static_switch<float, false, false, KIND_C2R>(L, var, a, st);
}
cudaError_t launch_static_group_real_f32(int L, bool r2c, const PassArgs *items,
                                         const int2 *tile_map, long long ntiles,
                                         cudaStream_t st) {
  return r2c ? launch_static_group_switch<float, false, true, KIND_R2C>(L, items, tile_map, ntiles, st)
             : launch_static_group_switch<float, false, false, KIND_C2R>(L, items, tile_map, ntiles, st);
}
} // namespace b200fft
