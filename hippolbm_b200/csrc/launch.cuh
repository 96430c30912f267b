// launch.cuh -- host-side launch of the step kernel for one (storage, compute) type.
// Each precision tier is its own translation unit so that the strict FP64 tier can be
// compiled without FMA contraction (--fmad=false) while the others use FMA.
#pragma once
#include <cuda_runtime.h>

#include "lbm_step_vec.cuh"

namespace hlbm {

// Geometry of a step launch: x along threadIdx.x (coalesced SoA rows), y on threadIdx.y,
// z on blockIdx.z.  256 threads per block.
inline void step_geometry(const StepPlan& p, dim3& grid, dim3& block) {
  int bx = 128;
  if (p.nx < 128) bx = ((p.nx + 31) / 32) * 32;
  int by = 256 / bx;
  block = dim3(bx, by, 1);
  grid = dim3((p.nx + bx - 1) / bx, (p.ny + by - 1) / by, p.nz);
}

template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int MINB>
cudaError_t launch_one(const void* fin, void* fout, const int8_t* flags, const StepPlan& p, cudaStream_t s) {
  dim3 grid, block;
  step_geometry(p, grid, block);
  k_step<S, R, STRICT, MODE, WALLS, true, MINB>
      <<<grid, block, 0, s>>>(static_cast<const S*>(fin), static_cast<S*>(fout), flags, p);
  return cudaGetLastError();
}

// nodes per thread of the vectorised kernel: one 8-byte vector per direction plane for the
// 4- and 2-byte storage types (float2, 4 x FP16/BF16); FP64 uses double2
template <typename S>
constexpr int vec_npt() {
  return sizeof(S) == 8 ? 2 : (sizeof(S) == 4 ? 2 : 4);
}

template <typename S>
bool vec_eligible(const StepPlan& p, int walls) {
  constexpr int NPT = vec_npt<S>();
  return !walls && p.nx % NPT == 0 && p.nx / NPT >= 32;
}

inline void vec_geometry(const StepPlan& p, int npt, int block_x, dim3& grid, dim3& block) {
  const int nvec = p.nx / npt;
  int bx = block_x > 0 ? block_x : 128;
  const int rounded = ((nvec + 31) / 32) * 32;
  if (rounded < bx) bx = rounded;
  const int by = 256 / bx > 0 ? 256 / bx : 1;
  block = dim3(bx, by, 1);
  grid = dim3((nvec + bx - 1) / bx, (p.ny + by - 1) / by, p.nz);
}

template <typename S, typename R, bool STRICT, int MODE, int MINB>
cudaError_t launch_vec(const void* fin, void* fout, const int8_t* flags, const StepPlan& p, cudaStream_t s) {
  constexpr int NPT = vec_npt<S>();
  dim3 grid, block;
  vec_geometry(p, NPT, 0, grid, block);
  k_step_vec<S, R, STRICT, MODE, NPT, MINB>
      <<<grid, block, 0, s>>>(static_cast<const S*>(fin), static_cast<S*>(fout), flags, p);
  return cudaGetLastError();
}

// Step kernel variants: variant % 2 selects the kernel (0: one node per thread, 1: vectorised
// when eligible), variant / 2 the occupancy target: at least 1, 2 or 3 blocks of 256 threads per
// SM (__launch_bounds__ minimum blocks, which caps registers at 255, 128 or 85 per thread).
constexpr int NUM_VARIANTS = 6;

template <typename S, typename R, bool STRICT, int MINB>
cudaError_t launch_minb(int mode, int walls, bool vec, const void* fin, void* fout, const int8_t* flags,
                        const StepPlan& p, cudaStream_t s) {
  if (vec) {
    if (mode == MODE_PROLOGUE) return launch_vec<S, R, STRICT, MODE_PROLOGUE, MINB>(fin, fout, flags, p, s);
    if (mode == MODE_FUSED) return launch_vec<S, R, STRICT, MODE_FUSED, MINB>(fin, fout, flags, p, s);
    return launch_vec<S, R, STRICT, MODE_FINISH, MINB>(fin, fout, flags, p, s);
  }
  if (mode == MODE_PROLOGUE)
    return walls ? launch_one<S, R, STRICT, MODE_PROLOGUE, true, MINB>(fin, fout, flags, p, s)
                 : launch_one<S, R, STRICT, MODE_PROLOGUE, false, MINB>(fin, fout, flags, p, s);
  if (mode == MODE_FUSED)
    return walls ? launch_one<S, R, STRICT, MODE_FUSED, true, MINB>(fin, fout, flags, p, s)
                 : launch_one<S, R, STRICT, MODE_FUSED, false, MINB>(fin, fout, flags, p, s);
  return walls ? launch_one<S, R, STRICT, MODE_FINISH, true, MINB>(fin, fout, flags, p, s)
               : launch_one<S, R, STRICT, MODE_FINISH, false, MINB>(fin, fout, flags, p, s);
}

template <typename S, typename R, bool STRICT>
cudaError_t launch_step(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                        cudaStream_t s, int variant) {
  const bool vec = (variant % 2) == 1 && vec_eligible<S>(p, walls);
  switch (variant / 2) {
    case 0: return launch_minb<S, R, STRICT, 1>(mode, walls, vec, fin, fout, flags, p, s);
    case 1: return launch_minb<S, R, STRICT, 2>(mode, walls, vec, fin, fout, flags, p, s);
    default: return launch_minb<S, R, STRICT, 3>(mode, walls, vec, fin, fout, flags, p, s);
  }
}

// one entry per precision tier (defined in step_*.cu)
cudaError_t step_f64_strict(int mode, int walls, const void* fin, void* fout, const int8_t* flags,
                            const StepPlan& p, cudaStream_t s, int variant);
cudaError_t step_f64(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant);
cudaError_t step_f32(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant);
cudaError_t step_f16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant);
cudaError_t step_bf16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                      cudaStream_t s, int variant);

}  // namespace hlbm
