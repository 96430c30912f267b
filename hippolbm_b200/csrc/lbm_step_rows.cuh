// lbm_step_rows.cuh -- the fused step of one lattice as a row pipeline: bulk copies of whole
// source rows into shared memory, node pairs updated from there in packed FP32.
//
// Work is a list of tiles, each `rows` consecutive x-rows (y0 .. y0 + rows - 1) of one z-plane,
// at most 128 nodes per consumer warp.  Warp 0 of a CTA produces: for every tile of its share, lane
// I (< 19) issues the cp.async.bulk copies of direction I's source rows (y - e_y, z - e_z; periodic
// images, or the node's own plane opp(I) where the source lies outside a non-periodic face) into a
// stage, and lane 19 copies the tile's flag bytes; all complete on the stage's `full` mbarrier.
// The other warps consume: each thread takes four consecutive nodes of a row (the same row and
// columns in every tile), reads every direction's values for them from the stage -- one base
// address with a compile-time offset per direction; the x-shift of a pull is an offset in the row
// (two aligned words and a byte permute for e_x = +-1), the row ends wrap inside the row or, on a
// non-periodic x face, bounce back with one global load -- and releases the stage at once (the
// producer refills it while the collisions run).  It then collides the two node pairs in packed
// FP32, rounds them (16-bit tiers: stochastic rounding into packed words) and stores straight to
// global memory with one 8- or 16-byte store per direction.  STAGES tiles are in flight while the
// consumers compute, so memory latency is off the consumers' path and few registers hold data.
//
// Like the vectorised kernel it applies no boundary operator (the face pass follows) and no wall
// test (the wall fix-up follows on lattices with wall obstacles), and takes fused steps only.
// Copies are plain (non-multicast) bulk loads of this GPU's own memory; every wait is bounded.
#pragma once
#include <cuda_runtime.h>

#include "lbm_step_tma.cuh"
#include "lbm_step_vec.cuh"

namespace hlbm {

constexpr int ROWS_NODES_PER_THREAD = 4;  // two node pairs

// Consumer warps and CTAs per SM of the two variants (each CTA adds its producer warp):
// variant 8 runs two CTAs of 8 consumer warps per SM (96 registers a thread), variant 9 one CTA of
// 12 (128 registers a thread: 13 warps leave 4 per scheduler).  The register budget decides: the
// node-pair collision of 38 lanes of state plus the other pair's 19 staged words spills heavily
// at 96 registers, and 12 warps at 128 registers step a 512^3 lattice 1.1x (BGK) to 1.2x (MRT)
// faster than 16 at 96.
constexpr int rows_warps(int variant) { return variant == 8 ? 8 : 12; }
constexpr int rows_ctas_per_sm(int variant) { return variant == 8 ? 2 : 1; }
constexpr int rows_tile_nodes(int warps) { return warps * 32 * ROWS_NODES_PER_THREAD; }

// Geometry of the row pipeline for one lattice: `rows` per tile, stage bytes, tiles.
struct RowsGeometry {
  int rows = 0;
  int tiles_per_plane = 0;
  int ntiles = 0;
  size_t stage_bytes = 0;  // 19 direction blocks of tile-node values (rows * nx used), then the flag bytes
};

inline size_t rows_align128(size_t b) { return (b + 127) / 128 * 128; }

// Whether a lattice can take the row pipeline: a 16-bit tier, rows of whole 16-byte chunks of flag
// bytes (and so of populations) and no longer than a tile, 32-bit node offsets, and the pair
// kernels' plan conditions.
inline bool rows_eligible(const StepPlan& p, int bytes, int warps) {
  return bytes == 2 && p.nx % 16 == 0 && p.nx <= rows_tile_nodes(warps) && p.ncell <= int64_t(0xffffffffu) &&
         pair_kernels_apply(p, bytes);
}

inline RowsGeometry rows_geometry(const StepPlan& p, int bytes, int warps) {
  RowsGeometry g;
  g.rows = rows_tile_nodes(warps) / p.nx > 0 ? rows_tile_nodes(warps) / p.nx : 1;
  if (g.rows > p.ny) g.rows = p.ny;
  g.tiles_per_plane = (p.ny + g.rows - 1) / g.rows;
  g.ntiles = g.tiles_per_plane * p.nz;
  g.stage_bytes = rows_align128(size_t(Q + 1) * rows_tile_nodes(warps) * bytes);
  return g;
}

inline size_t rows_smem_bytes(int stages, const RowsGeometry& g) { return 128 + size_t(stages) * g.stage_bytes; }

// Lane I of the producer: the source rows of direction I for tile rows y0 .. y0 + rows - 1 of
// plane z, as runs that are contiguous in memory (a run ends at a periodic y wrap or where the
// rows change between pulled and bounced), one bulk copy per run.
template <typename S>
__device__ __forceinline__ void rows_issue_direction(const Planes<S>& pl, const StepPlan& p, int z, int y0,
                                                     int rows, S* dst, uint64_t* bar, int i) {
  const int ey = dir_ey(i), ez = dir_ez(i), O = dir_opp(i);
  const int nx = p.nx;
  const unsigned row_bytes = unsigned(nx) * unsigned(sizeof(S));
  int sz = z - ez;
  if (sz < 0 || sz >= p.nz) sz = p.periodic[2] ? (sz < 0 ? sz + p.nz : sz - p.nz) : z;
  int r = 0;
  while (r < rows) {
    if (row_bounces(p, y0 + r, z, ey, ez)) {  // every node of the row bounces back on itself
      int r1 = r;
      while (r1 + 1 < rows && row_bounces(p, y0 + r1 + 1, z, ey, ez)) r1++;
      const S* src = pl.in[O] + (uint32_t(z) * uint32_t(p.ny) + uint32_t(y0 + r)) * uint32_t(nx);
      bulk_copy(dst + size_t(r) * nx, src, unsigned(r1 - r + 1) * row_bytes, bar);
      r = r1 + 1;
      continue;
    }
    int sy = y0 + r - ey;
    sy = sy < 0 ? sy + p.ny : (sy >= p.ny ? sy - p.ny : sy);
    int r1 = r;
    while (r1 + 1 < rows && !row_bounces(p, y0 + r1 + 1, z, ey, ez) && sy + (r1 + 1 - r) < p.ny) r1++;
    const S* src = pl.in[i] + (uint32_t(sz) * uint32_t(p.ny) + uint32_t(sy)) * uint32_t(nx);
    bulk_copy(dst + size_t(r) * nx, src, unsigned(r1 - r + 1) * row_bytes, bar);
    r = r1 + 1;
  }
}

// The value of direction I that element x (0 <= x < nx) of a staged source row gives, as a raw
// 16-bit value or float; x outside the row wraps (periodic x) or is the node's own opp(I)
// population at xn (non-periodic x: on-node bounce-back), fetched from global memory.
template <typename S, int I>
__device__ __forceinline__ S rows_edge_value(const S* row, int x, int nx, const Planes<S>& pl, uint32_t own_row,
                                             int xn, const StepPlan& p) {
  if (x >= 0 && x < nx) return row[x];
  if (p.periodic[0]) return row[x < 0 ? x + nx : x - nx];
  return ld_stream(pl.in[D3Q19::opp(I)] + own_row + uint32_t(xn));
}

// Four consecutive values (nodes x0 .. x0 + 3) of direction I from its staged source row, as the
// packed words of the two node pairs (16-bit tiers) or as floats.
template <typename S, int I>
__device__ __forceinline__ void rows_read(const S* row, int x0, int nx, bool bounced, const Planes<S>& pl,
                                          uint32_t own_row, const StepPlan& p, uint32_t (&w)[2], float (&f)[4]) {
  constexpr int ex = D3Q19::ex[I];  // a bounced row holds the node's own values: no shift
  if constexpr (is_16bit<S>()) {
    const uint32_t* words = reinterpret_cast<const uint32_t*>(row);
    if (ex == 0 || bounced) {
      const uint2 v = *reinterpret_cast<const uint2*>(words + x0 / 2);
      w[0] = v.x;
      w[1] = v.y;
    } else if constexpr (ex == 1) {  // elements x0-1 .. x0+2
      const uint2 v = *reinterpret_cast<const uint2*>(words + x0 / 2);
      uint32_t lo;
      if (x0 > 0) {
        lo = words[x0 / 2 - 1];
      } else {
        const S e = rows_edge_value<S, I>(row, -1, nx, pl, own_row, 0, p);
        lo = uint32_t(PackedChunk<S, 2>::bits(e)) << 16;
      }
      w[0] = __byte_perm(lo, v.x, 0x5432);  // (x0-1, x0)
      w[1] = __byte_perm(v.x, v.y, 0x5432);  // (x0+1, x0+2)
    } else {  // ex == -1: elements x0+1 .. x0+4
      const uint2 v = *reinterpret_cast<const uint2*>(words + x0 / 2);
      uint32_t hi;
      if (x0 + 4 < nx) {
        hi = words[x0 / 2 + 2];
      } else {
        const S e = rows_edge_value<S, I>(row, nx, nx, pl, own_row, nx - 1, p);
        hi = uint32_t(PackedChunk<S, 2>::bits(e));
      }
      w[0] = __byte_perm(v.x, v.y, 0x5432);  // (x0+1, x0+2)
      w[1] = __byte_perm(v.y, hi, 0x5432);   // (x0+3, x0+4)
    }
    (void)f;
  } else {
    if (ex == 0 || bounced) {
      const float4 v = *reinterpret_cast<const float4*>(row + x0);
      f[0] = v.x;
      f[1] = v.y;
      f[2] = v.z;
      f[3] = v.w;
    } else {
      const float4 v = *reinterpret_cast<const float4*>(row + x0);
      if constexpr (ex == 1) {
        f[0] = x0 > 0 ? row[x0 - 1] : rows_edge_value<S, I>(row, -1, nx, pl, own_row, 0, p);
        f[1] = v.x;
        f[2] = v.y;
        f[3] = v.z;
      } else {
        f[0] = v.y;
        f[1] = v.z;
        f[2] = v.w;
        f[3] = x0 + 4 < nx ? row[x0 + 4] : rows_edge_value<S, I>(row, nx, nx, pl, own_row, nx - 1, p);
      }
    }
    (void)w;
  }
}

// rows_read for a group away from the row ends of a row that pulls from no bounced row: every
// value is in the staged row, no test.
template <typename S, int I>
__device__ __forceinline__ void rows_read_interior(const S* row, int x0, uint32_t (&w)[2], float (&f)[4]) {
  constexpr int ex = D3Q19::ex[I];
  if constexpr (is_16bit<S>()) {
    const uint32_t* words = reinterpret_cast<const uint32_t*>(row);
    const uint2 v = *reinterpret_cast<const uint2*>(words + x0 / 2);
    if constexpr (ex == 0) {
      w[0] = v.x;
      w[1] = v.y;
    } else if constexpr (ex == 1) {
      const uint32_t lo = words[x0 / 2 - 1];
      w[0] = __byte_perm(lo, v.x, 0x5432);
      w[1] = __byte_perm(v.x, v.y, 0x5432);
    } else {
      const uint32_t hi = words[x0 / 2 + 2];
      w[0] = __byte_perm(v.x, v.y, 0x5432);
      w[1] = __byte_perm(v.y, hi, 0x5432);
    }
    (void)f;
  } else {
    const float4 v = *reinterpret_cast<const float4*>(row + x0);
    if constexpr (ex == 0) {
      f[0] = v.x, f[1] = v.y, f[2] = v.z, f[3] = v.w;
    } else if constexpr (ex == 1) {
      f[0] = row[x0 - 1], f[1] = v.x, f[2] = v.y, f[3] = v.z;
    } else {
      f[0] = v.y, f[1] = v.z, f[2] = v.w, f[3] = row[x0 + 4];
    }
    (void)w;
  }
}

template <typename S, int COLL, int STAGES, int WARPS, int MINB>
__global__ void __launch_bounds__(32 * (WARPS + 1), MINB)
    k_step_rows(const __grid_constant__ Planes<S> pl, const int8_t* __restrict__ flags, const StepPlan p,
                RowsGeometry g, int* __restrict__ err, long long wait_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + STAGES;
  unsigned char* stages = smem_raw + 128;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nx = p.nx;
  // direction I's rows start at element I * TILE of a stage (an immediate offset from one base);
  // the tile's flag bytes follow the 19 blocks
  constexpr int TILE = rows_tile_nodes(WARPS);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  advance_seed<S, MODE_FUSED>(p);
  __syncthreads();

  if (warp == 0) {  // ------------------------------------------------------------ producer
    int k = 0;
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, k++) {
      const int s = k % STAGES;
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, wait_limit)) {
        if (lane == 0) atomicExch(err, TMA_ERR_TIMEOUT);
        break;
      }
      const int z = t / g.tiles_per_plane, y0 = (t - z * g.tiles_per_plane) * g.rows;
      const int rows = (p.ny - y0) < g.rows ? (p.ny - y0) : g.rows;
      unsigned char* st = stages + size_t(s) * g.stage_bytes;
      if (lane == 0)
        mbar_arrive_expect_tx(&full[s], unsigned(size_t(Q) * rows * nx * sizeof(S) + size_t(rows) * nx));
      __syncwarp();
      if (lane < Q) {
        rows_issue_direction<S>(pl, p, z, y0, rows, reinterpret_cast<S*>(st) + lane * TILE, &full[s],
                                lane);
      } else if (lane == Q) {
        bulk_copy(st + Q * TILE * sizeof(S), flags + (uint32_t(z) * uint32_t(p.ny) + uint32_t(y0)) * nx,
                  unsigned(rows * nx), &full[s]);
      }
    }
    // every copy issued must land before the CTA exits (bounded by the default limit)
    const int issued = k;
    for (int kk = issued - STAGES < 0 ? 0 : issued - STAGES; kk < issued; kk++)
      mbar_wait(&full[kk % STAGES], (kk / STAGES) & 1);
    return;
  }

  // ------------------------------------------------------------------------ consumers
  const int ctid = threadIdx.x - 32;
  const uint32_t seed = launch_seed<S>(p);
  // nx <= TILE, so a tile's groups of four nodes (rows * nx / 4 <= TILE / 4) are at most one per
  // consumer thread, and a thread takes the same row and columns of every tile
  const int groups_per_row = nx / ROWS_NODES_PER_THREAD;
  const int r = ctid / groups_per_row;
  const int x0 = (ctid - r * groups_per_row) * ROWS_NODES_PER_THREAD;
  const bool sr = is_16bit<S>() && p.rounding;
  int k = 0;
  for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, k++) {
    const int s = k % STAGES;
    if (!mbar_wait(&full[s], (k / STAGES) & 1, wait_limit)) {
      if (ctid == 0) atomicExch(err, TMA_ERR_TIMEOUT);
      return;
    }
    const int z = t / g.tiles_per_plane, y0 = (t - z * g.tiles_per_plane) * g.rows;
    const int rows = (p.ny - y0) < g.rows ? (p.ny - y0) : g.rows;
    const S* st = reinterpret_cast<const S*>(stages + size_t(s) * g.stage_bytes);
    const int8_t* sflags = reinterpret_cast<const int8_t*>(st + Q * TILE);
    const bool active = r < rows;
    const int y = y0 + r;
    const uint32_t own_row = (uint32_t(z) * uint32_t(p.ny) + uint32_t(y)) * uint32_t(nx);
    const uint32_t own = own_row + uint32_t(x0);
    // the directions whose source row lies outside a non-periodic y / z face (bounced rows)
    const bool oy0 = !p.periodic[1] && y == 0, oyl = !p.periodic[1] && y == p.ny - 1;
    const bool oz0 = !p.periodic[2] && z == 0, ozl = !p.periodic[2] && z == p.nz - 1;
    uint32_t fl4 = 0;
    uint32_t words[Q][2];
    float vals[Q][4];
    if (active) {
      fl4 = *reinterpret_cast<const uint32_t*>(sflags + size_t(r) * nx + x0);
      if (!(oy0 || oyl || oz0 || ozl) && x0 > 0 && x0 + ROWS_NODES_PER_THREAD < nx) {  // no bounce, no row end
        Unroll<0, Q>::run([&]<int I>() {
          rows_read_interior<S, I>(st + I * TILE + r * nx, x0, words[I], vals[I]);
        });
      } else {
        Unroll<0, Q>::run([&]<int I>() {
          constexpr int ey = D3Q19::ey[I], ez = D3Q19::ez[I];
          const bool bounced = (ey == 1 && oy0) || (ey == -1 && oyl) || (ez == 1 && oz0) || (ez == -1 && ozl);
          rows_read<S, I>(st + I * TILE + r * nx, x0, nx, bounced, pl, own_row, p, words[I],
                          vals[I]);
        });
      }
    }
    // every value this warp reads from the stage is in registers: release it, so the producer
    // refills it while the collisions run rather than after them
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (!active) continue;
    Unroll<0, 2>::run([&]<int J>() {
      const int8_t fa = int8_t(fl4 >> (16 * J)), fb = int8_t(fl4 >> (16 * J + 8));
      float2 v[Q];
      if constexpr (is_16bit<S>())
        Unroll<0, Q>::run([&]<int I>() { v[I] = unpack2<S>(words[I][J]); });
      else
        Unroll<0, Q>::run([&]<int I>() { v[I] = make_float2(vals[I][2 * J], vals[I][2 * J + 1]); });
      pair_update<S, MODE_FUSED, COLL>(v, p, fa, fb);
      if constexpr (is_16bit<S>()) {
        uint32_t h = 0, h2 = 0;
        if (sr) {
          h = node_hash(int64_t(own) + 2 * J, seed);
          h2 = second_hash(h);
        }
        pack_pair<S>(v, sr, h, h2, [&]<int I>(uint32_t w) { words[I][J] = w; });
      } else {
        Unroll<0, Q>::run([&]<int I>() {
          vals[I][2 * J] = v[I].x;
          vals[I][2 * J + 1] = v[I].y;
        });
      }
    });
    if constexpr (is_16bit<S>())
      Unroll<0, Q>::run([&]<int I>() { *reinterpret_cast<uint2*>(pl.out[I] + own) = make_uint2(words[I][0], words[I][1]); });
    else
      Unroll<0, Q>::run([&]<int I>() {
        *reinterpret_cast<float4*>(pl.out[I] + own) = make_float4(vals[I][0], vals[I][1], vals[I][2], vals[I][3]);
      });
  }
}

}  // namespace hlbm
