// launch.cuh -- host-side launch of the step kernel for one (storage, compute) type.
// Each precision tier is its own translation unit so that the strict FP64 tier can be
// compiled without FMA contraction (--fmad=false) while the others use FMA.
#pragma once
#include <cuda_runtime.h>

#include "lbm_step_rows.cuh"
#include "lbm_step_spans.cuh"
#include "lbm_step_tiles.cuh"
#include "lbm_step_tma.cuh"
#include "lbm_step_vec.cuh"

namespace hlbm {

// Geometry of a step launch: x along threadIdx.x (coalesced SoA rows), y on threadIdx.y,
// z on blockIdx.z; or, for a plan with `linear` set, 256 consecutive nodes of a z-plane per
// block and z on blockIdx.y.  256 threads per block.
inline void step_geometry(const StepPlan& p, dim3& grid, dim3& block) {
  if (p.linear) {
    block = dim3(256, 1, 1);
    grid = dim3(unsigned((int64_t(p.nx) * p.ny + 255) / 256), p.nz, 1);
    return;
  }
  int bx = 128;
  if (p.nx < 128) bx = ((p.nx + 31) / 32) * 32;
  int by = 256 / bx;
  block = dim3(bx, by, 1);
  grid = dim3((p.nx + bx - 1) / bx, (p.ny + by - 1) / by, p.nz);
}

// The face pass after a step kernel that left the boundary operators out: the nodes of the faces
// in p.face_mask, recomputed whole by the one-node step.
template <typename S, typename R, bool STRICT, int MODE, bool WALLS>
cudaError_t launch_faces(const S* fi, S* fo, const int8_t* flags, const StepPlan& p, cudaStream_t s) {
  const int faces = p.face_mask;
  if (MODE == MODE_PROLOGUE || faces == 0) return cudaSuccess;
  int64_t area = 0;
  for (int f = 0; f < 6; f++)
    if (faces >> f & 1) {
      const int64_t a = f < 2 ? int64_t(p.ny) * p.nz : (f < 4 ? int64_t(p.nx) * p.nz : int64_t(p.nx) * p.ny);
      area = a > area ? a : area;
    }
  if ((faces & 3) == 3 && 2 * int64_t(p.ny) * p.nz > area) area = 2 * int64_t(p.ny) * p.nz;  // x faces interleaved
  const dim3 fgrid(unsigned((area + 255) / 256), 6, 1);
  if (MODE == MODE_FUSED && p.collision == 0)
    k_faces<S, R, STRICT, MODE, WALLS, 0><<<fgrid, 256, 0, s>>>(fi, fo, flags, p, faces);
  else if (MODE == MODE_FUSED)
    k_faces<S, R, STRICT, MODE, WALLS, 1><<<fgrid, 256, 0, s>>>(fi, fo, flags, p, faces);
  else
    k_faces<S, R, STRICT, MODE, WALLS, 2><<<fgrid, 256, 0, s>>>(fi, fo, flags, p, faces);
  return cudaGetLastError();
}

template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int MINB>
cudaError_t launch_one(const void* fin, void* fout, const int8_t* flags, const StepPlan& p, cudaStream_t s) {
  dim3 grid, block;
  step_geometry(p, grid, block);
  const S* fi = static_cast<const S*>(fin);
  S* fo = static_cast<S*>(fout);
  if constexpr (is_16bit<S>()) {
    if (pairs_eligible(p)) {  // two nodes per thread, packed stores
      const int64_t plane = int64_t(p.nx) * p.ny;
      const dim3 pgrid(unsigned((plane / 2 + 255) / 256), p.nz, 1);
      if (MODE == MODE_FUSED && p.collision == 0)
        k_step_pairs<S, R, STRICT, MODE, WALLS, 0, MINB><<<pgrid, 256, 0, s>>>(fi, fo, flags, p);
      else if (MODE == MODE_FUSED)
        k_step_pairs<S, R, STRICT, MODE, WALLS, 1, MINB><<<pgrid, 256, 0, s>>>(fi, fo, flags, p);
      else
        k_step_pairs<S, R, STRICT, MODE, WALLS, 2, MINB><<<pgrid, 256, 0, s>>>(fi, fo, flags, p);
      if (cudaError_t e = cudaGetLastError()) return e;
      return launch_faces<S, R, STRICT, MODE, WALLS>(fi, fo, flags, p, s);
    }
  }
  if (MODE == MODE_FUSED && p.collision == 0)
    k_step<S, R, STRICT, MODE, WALLS, 0, MINB><<<grid, block, 0, s>>>(fi, fo, flags, p);
  else if (MODE == MODE_FUSED)
    k_step<S, R, STRICT, MODE, WALLS, 1, MINB><<<grid, block, 0, s>>>(fi, fo, flags, p);
  else
    k_step<S, R, STRICT, MODE, WALLS, 2, MINB><<<grid, block, 0, s>>>(fi, fo, flags, p);
  if (cudaError_t e = cudaGetLastError()) return e;
  if constexpr (face_pass_tier<S>()) return launch_faces<S, R, STRICT, MODE, WALLS>(fi, fo, flags, p, s);
  return cudaSuccess;
}

// nodes per thread of the vectorised kernel at occupancy target MINB (d3q19.cuh: vec_npt_bytes)
template <typename S, int MINB>
constexpr int vec_npt() {
  return vec_npt_bytes(int(sizeof(S)), MINB);
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
cudaError_t launch_vec(int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                       cudaStream_t s) {
  constexpr int NPT = vec_npt<S, MINB>();
  dim3 grid, block;
  vec_geometry(p, NPT, 0, grid, block);
  const S* fi = static_cast<const S*>(fin);
  S* fo = static_cast<S*>(fout);
  const Planes<S> pl = make_planes(fi, fo, p.stride);
  if (MODE == MODE_FUSED && p.collision == 0)
    k_step_vec<S, R, STRICT, MODE, NPT, 0, MINB><<<grid, block, 0, s>>>(pl, flags, p);
  else if (MODE == MODE_FUSED)
    k_step_vec<S, R, STRICT, MODE, NPT, 1, MINB><<<grid, block, 0, s>>>(pl, flags, p);
  else
    k_step_vec<S, R, STRICT, MODE, NPT, 2, MINB><<<grid, block, 0, s>>>(pl, flags, p);
  if (cudaError_t e = cudaGetLastError()) return e;
  if (cudaError_t e = launch_faces<S, R, STRICT, MODE, false>(fi, fo, flags, p, s)) return e;
  if (!walls || MODE == MODE_PROLOGUE) return cudaSuccess;
  const unsigned wgrid = unsigned((p.ncell + 255) / 256);
  if (MODE == MODE_FUSED && p.collision == 0)
    k_wall_fixup<S, R, STRICT, MODE, 0><<<wgrid, 256, 0, s>>>(fi, fo, flags, p);
  else if (MODE == MODE_FUSED)
    k_wall_fixup<S, R, STRICT, MODE, 1><<<wgrid, 256, 0, s>>>(fi, fo, flags, p);
  else
    k_wall_fixup<S, R, STRICT, MODE, 2><<<wgrid, 256, 0, s>>>(fi, fo, flags, p);
  return cudaGetLastError();
}

// Step kernel variants 0..5: variant % 2 selects the kernel (0: one node per thread, 1:
// vectorised when eligible, else one node per thread at 3 blocks/SM), variant / 2 the occupancy
// target: at least 1, 2 or 3 blocks of 256
// threads per SM (__launch_bounds__ minimum blocks, which caps registers at 255, 128 or 85 per
// thread).  Variants 6 and 7: the bulk-copy pipelined persistent kernel (lbm_step_tma.cuh), with
// tiles of about 512 (variant 6) or 1024 (variant 7) nodes; fused steps only, when eligible.
// Variants 8 and 9 (single lattices): the row pipeline of the 16-bit tiers (lbm_step_rows.cuh),
// two or one CTA per SM; fused steps only, when eligible, else variant 5.
constexpr int NUM_VARIANTS = 10;

// what the pipelined kernel needs besides the plan
struct TmaArgs {
  LatticeDesc* desc = nullptr;
  const Tile* tiles = nullptr;
  int ntiles = 0;
  int tile_elems = 0;  // elements of one direction in a stage
  int stages = 0;      // 0: not eligible
  int parity = 0;
  int* err = nullptr;
  int grid = 0;
  int ctas_per_sm = 1;
  long long seed = -1;  // step number of a single-lattice launch; -1: the descriptors' counters
  int ndesc = 0;        // descriptors whose counters a batched launch advances
  long long wait_limit = TMA_WAIT_LIMIT;  // polls before a pipeline wait gives up
  bool rows = false;  // single lattice: variants 8 and 9 are the row pipeline (batches: tile kernels)
  int sms = 148;      // SMs of the device
};

template <typename S, typename R, bool STRICT, int STAGES, bool WALLS, int MINB>
cudaError_t launch_tma_t(const TmaArgs& a, cudaStream_t s) {
  auto kern = k_step_tma<S, R, STRICT, STAGES, WALLS, MINB>;
  const size_t smem = tma_smem_bytes(STAGES, a.tile_elems, sizeof(S));
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  kern<<<a.grid, TMA_THREADS, smem, s>>>(a.desc, a.tiles, a.ntiles, a.tile_elems, a.parity, a.err, a.seed,
                                                 a.ndesc, a.wait_limit);
  return cudaGetLastError();
}

template <typename S, typename R, bool STRICT, bool WALLS, int MINB>
cudaError_t launch_tma_stages(const TmaArgs& a, cudaStream_t s) {
  switch (a.stages) {
    case 2: return launch_tma_t<S, R, STRICT, 2, WALLS, MINB>(a, s);
    case 3: return launch_tma_t<S, R, STRICT, 3, WALLS, MINB>(a, s);
    default: return launch_tma_t<S, R, STRICT, 4, WALLS, MINB>(a, s);
  }
}

// ctas_per_sm: 1 or 2 (the stages of two CTAs must fit one SM's shared memory)
template <typename S, typename R, bool STRICT>
cudaError_t launch_tma(const TmaArgs& a, int walls, int ctas_per_sm, cudaStream_t s) {
  if (ctas_per_sm == 2)
    return walls ? launch_tma_stages<S, R, STRICT, true, 2>(a, s) : launch_tma_stages<S, R, STRICT, false, 2>(a, s);
  return walls ? launch_tma_stages<S, R, STRICT, true, 1>(a, s) : launch_tma_stages<S, R, STRICT, false, 1>(a, s);
}

template <typename S, typename R, bool STRICT, int MINB>
cudaError_t launch_minb(int mode, int walls, bool vec, const void* fin, void* fout, const int8_t* flags,
                        const StepPlan& p, cudaStream_t s) {
  if (vec) {
    if (mode == MODE_PROLOGUE) return launch_vec<S, R, STRICT, MODE_PROLOGUE, MINB>(walls, fin, fout, flags, p, s);
    if (mode == MODE_FUSED) return launch_vec<S, R, STRICT, MODE_FUSED, MINB>(walls, fin, fout, flags, p, s);
    return launch_vec<S, R, STRICT, MODE_FINISH, MINB>(walls, fin, fout, flags, p, s);
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

// tile-list kernel of batches (variant 8: >= 3 CTAs per SM, 9: >= 2)
template <typename S, typename R, bool STRICT, bool WALLS>
cudaError_t launch_tiles_persistent(const TmaArgs& a, cudaStream_t s) {
  auto kern = k_step_tiles_persistent<S, R, STRICT, WALLS, 3>;
  static const int resident = [kern] {  // CTAs resident on the whole device
    int per_sm = 0, dev = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (per_sm > 0 ? per_sm : 1) * sms;
  }();
  int grid = resident;
  if (grid > a.ntiles) grid = a.ntiles;
  if (grid < 1) return cudaSuccess;
  kern<<<grid, 256, 0, s>>>(a.desc, a.tiles, a.ntiles, a.parity, a.seed, a.ndesc);
  return cudaGetLastError();
}

// variant 8: one CTA per tile; 9: persistent tile walk (3 CTAs of 256 threads per SM)
template <typename S, typename R, bool STRICT>
cudaError_t launch_tiles(const TmaArgs& a, int walls, int variant, cudaStream_t s) {
  if (variant == 9)
    return walls ? launch_tiles_persistent<S, R, STRICT, true>(a, s) : launch_tiles_persistent<S, R, STRICT, false>(a, s);
  if (walls) k_step_tiles<S, R, STRICT, true, 3><<<a.ntiles, 256, 0, s>>>(a.desc, a.tiles, a.parity, a.seed, a.ndesc);
  else k_step_tiles<S, R, STRICT, false, 3><<<a.ntiles, 256, 0, s>>>(a.desc, a.tiles, a.parity, a.seed, a.ndesc);
  return cudaGetLastError();
}

// The row pipeline (lbm_step_rows.cuh) for one lattice: variant 8 = two CTAs per SM, variant 9 =
// one CTA per SM with deeper staging; the face pass and (with wall obstacles) the wall fix-up
// follow.  Returns cudaErrorNotSupported when the lattice or the mode cannot take it.
inline int rows_stages(const RowsGeometry& g, int ctas_per_sm) {
  const size_t budget = size_t(227 * 1024) / size_t(ctas_per_sm) - 1024;
  const size_t fit = (budget - 128) / g.stage_bytes;
  return fit >= 4 ? 4 : int(fit);
}

template <typename S, int COLL, int STAGES, int WARPS, int MINB>
cudaError_t launch_rows_t(const Planes<S>& pl, const int8_t* flags, const StepPlan& p, const RowsGeometry& g,
                          const TmaArgs& a, cudaStream_t s) {
  auto kern = k_step_rows<S, COLL, STAGES, WARPS, MINB>;
  const size_t smem = rows_smem_bytes(STAGES, g);
  if (cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) return e;
  const int grid = g.ntiles < a.sms * MINB ? g.ntiles : a.sms * MINB;
  kern<<<grid, 32 * (WARPS + 1), smem, s>>>(pl, flags, p, g, a.err, a.wait_limit);
  return cudaGetLastError();
}

template <typename S, int COLL, int WARPS, int MINB>
cudaError_t launch_rows_stages(int stages, const Planes<S>& pl, const int8_t* flags, const StepPlan& p,
                               const RowsGeometry& g, const TmaArgs& a, cudaStream_t s) {
  if (stages >= 4) return launch_rows_t<S, COLL, 4, WARPS, MINB>(pl, flags, p, g, a, s);
  if (stages == 3) return launch_rows_t<S, COLL, 3, WARPS, MINB>(pl, flags, p, g, a, s);
  return launch_rows_t<S, COLL, 2, WARPS, MINB>(pl, flags, p, g, a, s);
}

// The span pipeline (lbm_step_spans.cuh) with the shape of variant 8 or 9; its stage count is the
// one the variant's stage size allows (3 stages of 60 KB at one CTA per SM, 2 of 40 KB at two).
constexpr size_t spans_stage_bytes(int warps) {
  return (size_t(Q) * (spans_tile_nodes(warps) + 8) * 2 + size_t(spans_tile_nodes(warps)) + 127) / 128 * 128;
}
constexpr int spans_stage_count(int variant) {
  const size_t budget = size_t(227 * 1024) / size_t(rows_ctas_per_sm(variant)) - 1024;
  const size_t fit = (budget - 128) / spans_stage_bytes(rows_warps(variant));
  return fit >= 4 ? 4 : int(fit);
}
static_assert(spans_stage_count(8) >= 2 && spans_stage_count(9) >= 2, "span pipeline stages must fit");

template <typename S, int COLL, int VARIANT>
cudaError_t launch_spans_t(const Planes<S>& pl, const int8_t* flags, const StepPlan& p, const SpansGeometry& g,
                           const TmaArgs& a, cudaStream_t s) {
  constexpr int WARPS = rows_warps(VARIANT), MINB = rows_ctas_per_sm(VARIANT), STAGES = spans_stage_count(VARIANT);
  auto kern = k_step_spans<S, COLL, STAGES, WARPS, MINB>;
  const size_t smem = spans_smem_bytes(STAGES, g);
  if (cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) return e;
  const int grid = g.ntiles < a.sms * MINB ? g.ntiles : a.sms * MINB;
  kern<<<grid, 32 * (WARPS + 1), smem, s>>>(pl, flags, p, g, a.err, a.wait_limit);
  return cudaGetLastError();
}

// Which pipeline a fused step of `variant` (8 or 9) runs on the lattice: 1 the row pipeline (rows
// of whole 16-byte chunks), 2 the span pipeline (any other row length), 0 neither.
inline int pipeline_kind(const StepPlan& p, int variant, int bytes) {
  if (rows_eligible(p, bytes, rows_warps(variant)) &&
      rows_stages(rows_geometry(p, bytes, rows_warps(variant)), rows_ctas_per_sm(variant)) >= 2)
    return 1;
  if (spans_eligible(p, bytes)) return 2;
  return 0;
}

template <typename S, typename R, bool STRICT>
cudaError_t launch_rows(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                        cudaStream_t s, int variant, const TmaArgs& a) {
  if constexpr (!is_16bit<S>()) {
    return cudaErrorNotSupported;
  } else {
    const int kind = mode == MODE_FUSED ? pipeline_kind(p, variant, int(sizeof(S))) : 0;
    if (kind == 0) return cudaErrorNotSupported;
    const S* fi = static_cast<const S*>(fin);
    S* fo = static_cast<S*>(fout);
    const Planes<S> pl = make_planes(fi, fo, p.stride);
    cudaError_t e;
    if (kind == 1) {
      const int ctas = rows_ctas_per_sm(variant);
      const RowsGeometry g = rows_geometry(p, int(sizeof(S)), rows_warps(variant));
      const int stages = rows_stages(g, ctas);
      if (variant == 8)
        e = p.collision == 0 ? launch_rows_stages<S, 0, rows_warps(8), rows_ctas_per_sm(8)>(stages, pl, flags, p, g, a, s)
                             : launch_rows_stages<S, 1, rows_warps(8), rows_ctas_per_sm(8)>(stages, pl, flags, p, g, a, s);
      else
        e = p.collision == 0 ? launch_rows_stages<S, 0, rows_warps(9), rows_ctas_per_sm(9)>(stages, pl, flags, p, g, a, s)
                             : launch_rows_stages<S, 1, rows_warps(9), rows_ctas_per_sm(9)>(stages, pl, flags, p, g, a, s);
    } else {
      const SpansGeometry g = spans_geometry(p, rows_warps(variant));
      if (variant == 8)
        e = p.collision == 0 ? launch_spans_t<S, 0, 8>(pl, flags, p, g, a, s) : launch_spans_t<S, 1, 8>(pl, flags, p, g, a, s);
      else
        e = p.collision == 0 ? launch_spans_t<S, 0, 9>(pl, flags, p, g, a, s) : launch_spans_t<S, 1, 9>(pl, flags, p, g, a, s);
    }
    if (e) return e;
    if ((e = launch_faces<S, R, STRICT, MODE_FUSED, false>(fi, fo, flags, p, s))) return e;
    if (!walls) return cudaSuccess;
    const unsigned wgrid = unsigned((p.ncell + 255) / 256);
    if (p.collision == 0)
      k_wall_fixup<S, R, STRICT, MODE_FUSED, 0><<<wgrid, 256, 0, s>>>(fi, fo, flags, p);
    else
      k_wall_fixup<S, R, STRICT, MODE_FUSED, 1><<<wgrid, 256, 0, s>>>(fi, fo, flags, p);
    return cudaGetLastError();
  }
}

// Whether a single-lattice launch of `variant` in `mode` runs the row or span pipeline; otherwise
// variants 8 and 9 run variant 5.
inline bool rows_runs(const StepPlan& p, int variant, int mode, int bytes) {
  return variant >= 8 && mode == MODE_FUSED && pipeline_kind(p, variant, bytes) != 0;
}

template <typename S, typename R, bool STRICT>
cudaError_t launch_step(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                        cudaStream_t s, int variant, const TmaArgs& tma) {
  if (variant >= 8 && tma.rows) {
    if (rows_runs(p, variant, mode, int(sizeof(S))))
      return launch_rows<S, R, STRICT>(mode, walls, fin, fout, flags, p, s, variant, tma);
    variant = 5;
  }
  if (variant >= 8) return launch_tiles<S, R, STRICT>(tma, walls, variant, s);
  if (variant >= 6) {
    if (mode == MODE_FUSED && tma.stages >= 2) return launch_tma<S, R, STRICT>(tma, walls, tma.ctas_per_sm, s);
    variant = 4;
  }
  const bool vec = (variant % 2) == 1 && vec_eligible_bytes(p, walls, int(sizeof(S)), variant);
  if ((variant % 2) == 1 && !vec) variant = 4;  // no vectorised kernel for this lattice: 3 CTAs/SM scalar
  switch (variant / 2) {
    case 0: return launch_minb<S, R, STRICT, 1>(mode, walls, vec, fin, fout, flags, p, s);
    case 1: return launch_minb<S, R, STRICT, 2>(mode, walls, vec, fin, fout, flags, p, s);
    default: return launch_minb<S, R, STRICT, 3>(mode, walls, vec, fin, fout, flags, p, s);
  }
}

// one entry per precision tier (defined in step_*.cu)
cudaError_t step_f64_strict(int mode, int walls, const void* fin, void* fout, const int8_t* flags,
                            const StepPlan& p, cudaStream_t s, int variant, const TmaArgs& tma);
cudaError_t step_f64(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma);
cudaError_t step_f32(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma);
cudaError_t step_f16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                     cudaStream_t s, int variant, const TmaArgs& tma);
cudaError_t step_bf16(int mode, int walls, const void* fin, void* fout, const int8_t* flags, const StepPlan& p,
                      cudaStream_t s, int variant, const TmaArgs& tma);

}  // namespace hlbm
