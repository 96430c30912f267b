// lbm_step_tiles.cuh -- the fused step over a list of tiles of many lattices (batches).
//
// One CTA per tile; a tile is `rows` consecutive x-rows (one z plane) of one lattice of the
// batch.  The CTA stages its lattice's plan in shared memory, then every thread advances nodes
// of the tile with the per-node step of lbm_step.cuh (direct pulls from global memory, the same
// arithmetic as the single-lattice kernel).  A lattice whose descriptor carries the prologue flag
// takes its first step (collide S_0, no pull) in the same launch.
#pragma once
#include "lbm_step_tma.cuh"

namespace hlbm {

template <typename S, typename R, bool STRICT, bool WALLS, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_step_tiles(LatticeDesc* __restrict__ lats, const Tile* __restrict__ tiles, int parity, long long seed,
                 int ndesc) {
  __shared__ StepPlan splan;
  advance_step_numbers(lats, ndesc, seed, parity, threadIdx.x, blockDim.x);
  const Tile tl = tiles[blockIdx.x];
  const LatticeDesc L = lats[tl.x];
  const uint32_t* src = reinterpret_cast<const uint32_t*>(L.plan);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&splan);
  for (int w = threadIdx.x; w < int(sizeof(StepPlan) / 4); w += blockDim.x) dst[w] = src[w];
  __syncthreads();
  if (threadIdx.x == 0) splan.seed = launch_step_number(L, seed, parity);
  __syncthreads();
  const StepPlan& p = splan;
  const S* fin = static_cast<const S*>(L.f[L.cur ^ parity]);
  S* fout = static_cast<S*>(L.f[(L.cur ^ parity) ^ 1]);
  const int nodes = tl.w * p.nx;
  for (int n = threadIdx.x; n < nodes; n += blockDim.x) {
    const int r = n / p.nx, x = n - r * p.nx;
    if (L.prologue)
      node_step<S, R, STRICT, MODE_PROLOGUE, WALLS, 2>(fin, fout, L.flags, p, x, tl.z + r, tl.y);
    else
      node_step<S, R, STRICT, MODE_FUSED, WALLS, 2>(fin, fout, L.flags, p, x, tl.z + r, tl.y);
  }
}

}  // namespace hlbm
