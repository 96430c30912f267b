// FP32 compute, FP32 population storage.
#include "launch.cuh"
namespace hlbm {
cudaError_t step_f32(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma) {
  return launch_step<float, float, false>(mode, walls, fin, fout, flags, p, s, variant, tma);
}
}  // namespace hlbm
