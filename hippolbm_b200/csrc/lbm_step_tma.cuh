// lbm_step_tma.cuh -- the fused step as a persistent kernel fed by bulk asynchronous copies.
//
// Work is a packed list of tiles; a tile is `rows` consecutive x-rows (y0 .. y0+rows-1 at one z)
// of one lattice, so the same kernel advances a single lattice or a batch of lattices of
// different sizes and plans.  Warp 0 produces: for each tile, lane i issues the cp.async.bulk
// copies of the source rows (y - e_iy, z - e_iz) of population plane i into a shared-memory
// stage (rows whose source lies outside a non-periodic face are copied from the node's own
// plane opp(i) instead: on-node bounce-back); the copies complete on the stage's `full`
// mbarrier.  Warps 1..8 consume: they wait on `full`, compute the tile, and release the stage on
// its `empty` mbarrier.  STAGES tiles are in flight while the consumers compute the oldest one,
// so HBM stays busy independently of how many warps are resident.  The x-shift of a pull becomes a shared-memory
// offset (periodic wrap inside the row); the per-node work (boundary operators, start_iteration
// boxes, macro variables, BGK / MRT) is the one of lbm_step.cuh, and results go straight to
// global memory with coalesced stores.
//
// Copies are plain (non-multicast) bulk loads of this GPU's own memory.  Every mbarrier wait is
// bounded: a work wait gives up after `wait_limit` polls (about a second by default), records an
// error code in *err, and its warp returns; the producer then waits (bounded by the default
// limit) for the copies it has in flight before the CTA exits.
#pragma once
#include <cuda_runtime.h>

#include "lbm_step.cuh"

namespace hlbm {

// One lattice of a batch: its plan (device memory) and its two population buffers.
struct LatticeDesc {
  const StepPlan* plan;
  void* f[2];
  const int8_t* flags;
  int32_t cur;       // f[cur ^ parity] is read, the other written
  int32_t prologue;  // 1: the buffer read holds S_0; collide it without streaming (first step)
  uint32_t step[2];  // step number of the next launch of each parity (batched launches)
  uint32_t pad[2];
};

// Step number (rounding salt) of a launch: `seed` when the host passes one (>= 0), else the
// lattice's own counter for this parity.  A batched launch also advances the counters: block 0
// writes step[parity ^ 1] = step[parity] + 1, which no block of this launch reads.
__device__ __forceinline__ uint32_t launch_step_number(const LatticeDesc& L, long long seed, int parity) {
  return seed >= 0 ? uint32_t(seed) : L.step[parity];
}
__device__ __forceinline__ void advance_step_numbers(LatticeDesc* lats, int ndesc, long long seed, int parity,
                                                     int tid, int nthreads) {
  if (seed >= 0 || blockIdx.x != 0) return;
  for (int m = tid; m < ndesc; m += nthreads) lats[m].step[parity ^ 1] = lats[m].step[parity] + 1u;
}

// tile: {lattice, z, y0, rows}
using Tile = int4;

constexpr long long TMA_WAIT_LIMIT = 20000000;  // polls before a wait gives up (and at most ~2 s)
constexpr int TMA_ERR_TIMEOUT = 1;

// direction components for loops indexed at run time: 2 bits per direction (component + 1)
constexpr uint64_t pack_component(const int* e) {
  uint64_t v = 0;
  for (int i = 0; i < Q; i++) v |= uint64_t(e[i] + 1) << (2 * i);
  return v;
}
constexpr uint64_t EY_PACKED = pack_component(D3Q19::ey);
constexpr uint64_t EZ_PACKED = pack_component(D3Q19::ez);
__device__ __forceinline__ int dir_ey(int i) { return int((EY_PACKED >> (2 * i)) & 3u) - 1; }
__device__ __forceinline__ int dir_ez(int i) { return int((EZ_PACKED >> (2 * i)) & 3u) - 1; }
__device__ __forceinline__ int dir_opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

__host__ __device__ constexpr size_t tma_head_bytes() { return 128 + ((sizeof(StepPlan) + 127) / 128) * 128; }

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase with the given parity; false if it did not complete within `limit` polls or
// about two seconds.  The first poll is a non-blocking test; the others are `try_wait`, which
// suspends the thread in hardware until the phase completes or about a microsecond passes, so a
// waiting warp takes no issue slots from the warps that compute.
constexpr unsigned long long MBAR_WAIT_NS = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit = TMA_WAIT_LIMIT) {
  const unsigned a = smem_addr(bar);
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  if (done) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 1; it < limit; it++) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(1000u)
        : "memory");
    if (done) return true;
    if ((it & 63) == 0 && global_ns() - t0 > MBAR_WAIT_NS) return false;
  }
  return false;
}

// bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) global -> shared
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr int TMA_CONSUMER_WARPS = 8;
constexpr int TMA_THREADS = 32 * (TMA_CONSUMER_WARPS + 1);  // warp 0 produces, warps 1..8 consume

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// true when the pull of direction (ey, ez) for row y, plane z comes from outside a non-periodic
// face: that row of the stage holds the node's own plane opp(i) (on-node bounce-back)
__device__ __forceinline__ bool row_bounces(const StepPlan& p, int y, int z, int ey, int ez) {
  const int sy = y - ey, sz = z - ez;
  return ((sz < 0 || sz >= p.nz) && !p.periodic[2]) || ((sy < 0 || sy >= p.ny) && !p.periodic[1]);
}

// Lane i (< Q) of the producer warp copies direction i of one tile: runs of source rows that are
// contiguous in memory, one bulk copy per run.  The stage's byte count is registered beforehand.
template <typename S>
__device__ __forceinline__ void issue_direction(const LatticeDesc& L, const StepPlan& p, int parity, Tile t,
                                                S* stage, int tile_elems, uint64_t* bar, int i) {
  const int z = t.y, y0 = t.z, rows = t.w, nx = p.nx;
  const S* fin = static_cast<const S*>(L.f[L.cur ^ parity]);
  const size_t row_bytes = size_t(nx) * sizeof(S);
  S* dst = stage + size_t(i) * tile_elems;
  if (L.prologue) {  // first step: this tile's own rows of plane i, no pull
    bulk_copy(dst, fin + size_t(i) * p.stride + (size_t(z) * p.ny + y0) * nx, unsigned(rows * row_bytes), bar);
    return;
  }
  const int ey = dir_ey(i), ez = dir_ez(i), O = dir_opp(i);
  int sz = z - ez;
  if (sz < 0 || sz >= p.nz) sz = p.periodic[2] ? (sz < 0 ? sz + p.nz : sz - p.nz) : z;
  int r = 0;
  while (r < rows) {
    if (row_bounces(p, y0 + r, z, ey, ez)) {
      int r1 = r;
      while (r1 + 1 < rows && row_bounces(p, y0 + r1 + 1, z, ey, ez)) r1++;
      const S* src = fin + size_t(O) * p.stride + (size_t(z) * p.ny + (y0 + r)) * nx;
      bulk_copy(dst + size_t(r) * nx, src, unsigned((r1 - r + 1) * row_bytes), bar);
      r = r1 + 1;
      continue;
    }
    int sy = y0 + r - ey;
    sy = sy < 0 ? sy + p.ny : (sy >= p.ny ? sy - p.ny : sy);
    int r1 = r;
    while (r1 + 1 < rows && !row_bounces(p, y0 + r1 + 1, z, ey, ez) && sy + (r1 + 1 - r) < p.ny) r1++;
    const S* src = fin + size_t(i) * p.stride + (size_t(sz) * p.ny + sy) * nx;
    bulk_copy(dst + size_t(r) * nx, src, unsigned((r1 - r + 1) * row_bytes), bar);
    r = r1 + 1;
  }
}

template <typename S, typename R, bool STRICT, int STAGES, bool WALLS, int MINB>
__global__ void __launch_bounds__(TMA_THREADS, MINB)
    k_step_tma(LatticeDesc* __restrict__ lats, const Tile* __restrict__ tiles, int ntiles, int tile_elems,
               int parity, int* __restrict__ err, long long seed, int ndesc, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + STAGES;
  StepPlan* splan = reinterpret_cast<StepPlan*>(smem_raw + 128);
  S* stages = reinterpret_cast<S*>(smem_raw + tma_head_bytes());
  const size_t stage_elems = size_t(Q) * tile_elems;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TMA_CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == 0) {  // ------------------------------------------------------------ producer
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
      const int s = k % STAGES;
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, wait_limit)) {  // consumers released s
        if (lane == 0) atomicExch(err, TMA_ERR_TIMEOUT);
        break;
      }
      const Tile tl = tiles[t];
      const LatticeDesc L = lats[tl.x];
      const StepPlan& p = *L.plan;
      if (lane == 0) mbar_arrive_expect_tx(&full[s], unsigned(Q * tl.w * p.nx * sizeof(S)));
      __syncwarp();
      if (lane < Q) issue_direction<S>(L, p, parity, tl, stages + s * stage_elems, tile_elems, &full[s], lane);
    }
    // every copy issued must land before the CTA exits (bounded by the full limit, whatever the
    // work waits' limit: the copies of a stage land within microseconds)
    const int issued = k;
    for (int kk = issued - STAGES < 0 ? 0 : issued - STAGES; kk < issued; kk++)
      mbar_wait(&full[kk % STAGES], (kk / STAGES) & 1);
    return;
  }

  // ------------------------------------------------------------------------ consumers
  const int ctid = threadIdx.x - 32;
  constexpr int NC = 32 * TMA_CONSUMER_WARPS;
  advance_step_numbers(lats, ndesc, seed, parity, ctid, NC);
  int plan_of = -1;
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
    const int s = k % STAGES;
    const Tile tl = tiles[t];
    if (tl.x != plan_of) {  // stage this lattice's plan in shared memory (uniform over consumers)
      asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory");
      const uint32_t* src = reinterpret_cast<const uint32_t*>(lats[tl.x].plan);
      uint32_t* dst = reinterpret_cast<uint32_t*>(splan);
      for (int w = ctid; w < int(sizeof(StepPlan) / 4); w += NC) dst[w] = src[w];
      asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory");
      if (ctid == 0) splan->seed = launch_step_number(lats[tl.x], seed, parity);
      asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory");
      plan_of = tl.x;
    }
    if (!mbar_wait(&full[s], (k / STAGES) & 1, wait_limit)) {
      if (ctid == 0) atomicExch(err, TMA_ERR_TIMEOUT);
      return;
    }
    const StepPlan& p = *splan;
    const LatticeDesc L = lats[tl.x];
    const S* stage = stages + s * stage_elems;
    const S* fin = static_cast<const S*>(L.f[L.cur ^ parity]);
    S* fout = static_cast<S*>(L.f[(L.cur ^ parity) ^ 1]);
    const bool first = L.prologue != 0;
    const int nx = p.nx, ny = p.ny, nz = p.nz, z = tl.y, y0 = tl.z, rows = tl.w;
    const int nodes = rows * nx;
    const int64_t stride = p.stride;
    for (int n = ctid; n < nodes; n += NC) {
      const int r = n / nx, x = n - r * nx;
      const int y = y0 + r;
      const int64_t idx = (int64_t(z) * ny + y) * nx + x;
      const int8_t flag = L.flags[idx];
      if (WALLS && flag == FLAG_WALL) continue;
      R v[Q];
      Unroll<0, Q>::run([&]<int I>() {
        constexpr int ex = D3Q19::ex[I], ey = D3Q19::ey[I], ez = D3Q19::ez[I];
        constexpr int O = D3Q19::opp(I);
        const S* row = stage + size_t(I) * tile_elems + size_t(r) * nx;
        if (first) {  // own node, plane I
          v[I] = load_value<S, R, I>(row[x], p);
          return;
        }
        if (I != 0 && row_bounces(p, y, z, ey, ez)) {  // the stage row holds this node's plane opp(I)
          v[I] = load_value<S, R, O>(row[x], p);
          return;
        }
        int xs = x - ex;
        bool bounce = false;
        if (xs < 0 || xs >= nx) {
          if (p.periodic[0]) xs = xs < 0 ? xs + nx : xs - nx; else bounce = true;
        }
        if (WALLS && I != 0 && !bounce) {
          int sy = y - ey, sz = z - ez;
          sy = sy < 0 ? sy + ny : (sy >= ny ? sy - ny : sy);
          sz = sz < 0 ? sz + nz : (sz >= nz ? sz - nz : sz);
          bounce = L.flags[(int64_t(sz) * ny + sy) * nx + xs] == FLAG_WALL;
        }
        if (bounce)
          v[I] = load_value<S, R, O>(ld_stream(fin + O * stride + idx), p);
        else
          v[I] = load_value<S, R, I>(row[xs], p);
      });
      node_update<S, R, STRICT, MODE_FUSED, 2>(v, fin, idx, x, y, z, flag, p, !first, on_op_face(p, x, y, z));
      store_node<S, R, MODE_FUSED>(v, p, p.seed, idx, [&]<int I>(S s) { fout[I * stride + idx] = s; });
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
  }
}

// shared memory of one CTA: barriers (128 B), the staged plan, then the stages
inline size_t tma_smem_bytes(int stages, int tile_elems, size_t esize) {
  return tma_head_bytes() + size_t(stages) * Q * tile_elems * esize;
}

}  // namespace hlbm
