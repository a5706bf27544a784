// Specialised R2C (forward) and C2R (backward) row kernels, FP64.
#include "fs_launch.cuh"

namespace b200fft {
cudaError_t launch_static_r2c_f64(int L, int var, const PassArgs &a, cudaStream_t st) {
  return launch_static_switch<double, false, true, KIND_R2C>(L, var, a, st);
}
cudaError_t launch_static_c2r_f64(int L, int var, const PassArgs &a, cudaStream_t st) {
  return launch_static_switch<double, false, false, KIND_C2R>(L, var, a, st);
}
} // namespace b200fft
