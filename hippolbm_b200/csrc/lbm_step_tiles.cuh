// lbm_step_tiles.cuh -- the fused step over a list of tiles of many lattices (batches).
//
// A tile is `rows` consecutive x-rows (one z plane) of one lattice of the batch, about 256 nodes.
// Every thread advances nodes of a tile with the per-node step of lbm_step.cuh (direct pulls from
// global memory, the same arithmetic as the single-lattice kernel), with the tile's lattice plan
// staged in shared memory.  A lattice whose descriptor carries the prologue flag takes its first
// step (collide S_0, no pull) in the same launch.
//
// k_step_tiles_persistent: a grid sized to the resident CTAs, each CTA walking a contiguous range
// of the tile list (tiles are ordered by lattice, so a range crosses few lattices): the plan is
// staged only when the lattice changes and the next tile's entry is fetched while the current
// tile is computed, so no CTA start-up or plan copy sits in front of every 256 nodes.
// k_step_tiles: one CTA per tile.
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

template <typename S, typename R, bool STRICT, bool WALLS, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_step_tiles_persistent(LatticeDesc* __restrict__ lats, const Tile* __restrict__ tiles, int ntiles, int parity,
                            long long seed, int ndesc) {
  __shared__ StepPlan splan;
  advance_step_numbers(lats, ndesc, seed, parity, threadIdx.x, blockDim.x);
  const int per = (ntiles + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per;
  const int t1 = t0 + per < ntiles ? t0 + per : ntiles;
  int plan_of = -1;
  LatticeDesc L{};
  Tile next = t0 < t1 ? tiles[t0] : Tile{};
  for (int t = t0; t < t1; t++) {
    const Tile tl = next;
    if (t + 1 < t1) next = tiles[t + 1];
    if (tl.x != plan_of) {  // uniform over the CTA
      __syncthreads();      // every thread is done with the previous plan
      L = lats[tl.x];
      const uint32_t* src = reinterpret_cast<const uint32_t*>(L.plan);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&splan);
      for (int w = threadIdx.x; w < int(sizeof(StepPlan) / 4); w += blockDim.x) dst[w] = src[w];
      __syncthreads();
      if (threadIdx.x == 0) splan.seed = launch_step_number(L, seed, parity);
      __syncthreads();
      plan_of = tl.x;
    }
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
}

}  // namespace hlbm
