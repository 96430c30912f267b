// FP64 step with FMA contraction and reciprocal multiplies (the plain FP64 path).
#include "launch.cuh"
namespace hlbm {
cudaError_t step_f64(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma) {
  return launch_step<double, double, false>(mode, walls, fin, fout, flags, p, s, variant, tma);
}
}  // namespace hlbm
