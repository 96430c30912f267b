// FP64 step, reference operation order (compiled with --fmad=false: no contraction, true
// divisions), so that its populations equal the oracle's value for value.
#include "launch.cuh"
namespace hlbm {
cudaError_t step_f64_strict(int mode, int walls, const void* fin, void* fout, const int8_t* flags,
                            const StepPlan& p, cudaStream_t s, int variant, const TmaArgs& tma) {
  return launch_step<double, double, true>(mode, walls, fin, fout, flags, p, s, variant, tma);
}
}  // namespace hlbm
