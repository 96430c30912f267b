// FP32 compute, populations stored as FP16 deviations (f_i - w_i * rho0) * scale.
#include "launch.cuh"
namespace hlbm {
cudaError_t step_f16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma) {
  return launch_step<__half, float, false>(mode, walls, fin, fout, flags, p, s, variant, tma);
}
}  // namespace hlbm
