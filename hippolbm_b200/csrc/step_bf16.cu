// FP32 compute, populations stored as BF16 deviations (f_i - w_i * rho0) * scale.
#include "launch.cuh"
namespace hlbm {
cudaError_t step_bf16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                      cudaStream_t s, int variant, const TmaArgs& tma) {
  return launch_step<__nv_bfloat16, float, false>(mode, walls, fin, fout, flags, p, s, variant, tma);
}
}  // namespace hlbm
