// aux_kernels.cuh -- launchers for the non-step kernels (see aux_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "d3q19.cuh"

namespace hlbm {

enum ObstacleType : int32_t { OBS_NONE = -1, OBS_BALL = 0, OBS_WALL = 1, OBS_QUADRIC = 2 };

// Ball: a = {cx, cy, cz, r, r*r}; Wall: a = {min xyz, max xyz}; Quadric: a = Q row-major.
struct ObstacleDesc {
  int32_t type;
  double a[16];
};

cudaError_t launch_set_distribution(int prec, void* f, const StepPlan& p, const int lo[3], const int hi[3],
                                    double value, cudaStream_t s);
cudaError_t launch_double_couette(int prec, void* f, const StepPlan& p, int dim, const double uc[3],
                                  const double du[3], cudaStream_t s);
struct LatticeDesc;
cudaError_t launch_zero_gradient(int prec, const LatticeDesc* lats, int m, int face, int parity, const int n[3],
                                 cudaStream_t s);
cudaError_t launch_rasterize(int8_t* flags, const StepPlan& p, const int lo[3], const int hi[3], double dx,
                             const ObstacleDesc& o, cudaStream_t s);
cudaError_t launch_near_wall(const int8_t* flags, int8_t* near, const int n[3], const int periodic[3],
                             cudaStream_t s);
int stats_blocks(int64_t ncell);
cudaError_t launch_macro_stats(int prec, const void* f, const int8_t* flags, const StepPlan& p, double* rho,
                               double* u, double* partials, double* out3, cudaStream_t s);
cudaError_t launch_residual(int prec, const void* f, const int8_t* flags, const StepPlan& p, float* uprev, int first,
                            double* partials, double* out4, cudaStream_t s);
cudaError_t launch_moments(int prec, const void* f, const int8_t* flags, const StepPlan& p, double* partials,
                           double* out4, cudaStream_t s);
cudaError_t launch_wall_force(int prec, const void* fpost, const int8_t* flags, const StepPlan& p, double* partials,
                              double* out4, cudaStream_t s);
cudaError_t launch_plane_profile(int prec, const void* f, const int8_t* flags, const StepPlan& p, int dim,
                                 double ratio, double* out4n, cudaStream_t s);
cudaError_t launch_reencode(int prec, void* f, const StepPlan& old_plan, const StepPlan& new_plan, cudaStream_t s);
cudaError_t launch_decode(int prec, const void* f, double* out, int dir, const StepPlan& p, cudaStream_t s);
cudaError_t launch_encode(int prec, void* f, const double* in, int dir, const StepPlan& p, cudaStream_t s);

}  // namespace hlbm
