// lbm_step_spans.cuh -- the row pipeline for rows of any length: tiles are spans of the linear
// node index, bulk-copied per direction, node pairs updated from shared memory in packed FP32.
//
// The row pipeline (lbm_step_rows.cuh) stages whole x-rows, so it needs rows of whole 16-byte
// chunks (nx a multiple of 16).  This kernel takes any nx >= 4.  A tile is TILE consecutive node
// indices [t0, t0 + TILE) (t0 a multiple of TILE, TILE a multiple of 16).  Away from the faces the
// node n pulls direction I from n - d_I, d_I = (e_z ny + e_y) nx + e_x, so the tile's sources of
// direction I are one contiguous range [t0 - d_I, t0 - d_I + TILE).  Warp 0 produces: lane I
// bulk-copies that range, widened to 16-byte boundaries and clipped to the planes, into the stage's
// direction block I at the same offset modulo 8 elements; lane 19 copies the tile's flag bytes.
// Because t0 is a multiple of 8, the offset of the first value in block I, (-d_I) mod 8, is the
// same for every tile, so the host passes each direction's word offset and byte-permute selector
// and a consumer reads its four nodes of direction I as three aligned words and two permutes.
//
// A group of four nodes whose sources all lie inside the lattice (no node on a face, all in one
// row) reads only the stage.  In the other groups the nodes off the faces still read the stage;
// a face node either lies on a face the face pass recomputes (left for it) or pulls all its values
// from global memory with the one-node kernel's gather (periodic wrap, on-node bounce-back).
// Like the row pipeline it applies no boundary operator (the face pass follows), no wall test (the
// wall fix-up follows on lattices with wall obstacles), and takes fused steps of the 16-bit tiers
// only; the node pairs (n, n + 1), n even, and their random bits are those of every other kernel,
// so its results equal theirs bit for bit.  Copies are plain (non-multicast) bulk loads of this
// GPU's own memory; every wait is bounded.
#pragma once
#include <cuda_runtime.h>

#include "lbm_step_rows.cuh"

namespace hlbm {

// Geometry of the span pipeline for one lattice (computed on the host, passed by value).
struct SpansGeometry {
  int ntiles = 0;
  int block = 0;           // elements per direction block of a stage: TILE + 8
  size_t stage_bytes = 0;  // 19 direction blocks, then TILE flag bytes
  int64_t ncell8 = 0;      // copies of population planes end at most here (planes are padded to 128)
  int64_t ncell16 = 0;     // copies of flag bytes end at most here (the flags are padded to 128)
  int64_t d[Q];            // pull distance of direction I in the linear index
  uint32_t word[Q];        // 32-bit word of a stage holding the first value of direction I for node t0
  uint32_t sel[Q];         // __byte_perm selector: 0x3210 when that value is a low half-word, else 0x5432
  uint64_t mplane = 0, mnx = 0;  // ceil(2^64 / d) of the plane size and of nx: q = umul64hi(n, m)
};

constexpr int spans_tile_nodes(int warps) { return warps * 32 * ROWS_NODES_PER_THREAD; }

// Whether a lattice can take the span pipeline: a 16-bit tier, rows of at least one group of four
// nodes (a group then crosses at most one row end), 32-bit node indices, and the pair kernels'
// plan conditions.
inline bool spans_eligible(const StepPlan& p, int bytes) {
  return bytes == 2 && p.nx >= 4 && p.ncell <= int64_t(0xffffffffu) && pair_kernels_apply(p, bytes);
}

// ceil(2^64 / d) for 2 <= d < 2^32: then floor(n / d) = umul64hi(n, m) for every n < 2^32 (the
// product overshoots n / d by less than n / 2^64 < 1 / d).
inline uint64_t spans_magic(uint64_t d) {
  return ~uint64_t(0) / d + 1;  // floor((2^64 - 1) / d) + 1 = ceil(2^64 / d) when d is no power of two
}

inline SpansGeometry spans_geometry(const StepPlan& p, int warps) {
  SpansGeometry g;
  const int T = spans_tile_nodes(warps);
  g.ntiles = int((p.ncell + T - 1) / T);
  g.block = T + 8;
  g.stage_bytes = rows_align128(size_t(Q) * g.block * 2 + size_t(T));
  g.ncell8 = (p.ncell + 7) / 8 * 8;
  g.ncell16 = (p.ncell + 15) / 16 * 16;
  const int64_t plane = int64_t(p.nx) * p.ny;
  for (int i = 0; i < Q; i++) {
    g.d[i] = (int64_t(D3Q19::ez[i]) * p.ny + D3Q19::ey[i]) * p.nx + D3Q19::ex[i];
    const int off = int(((-g.d[i]) % 8 + 8) % 8);  // first value's element in its block
    g.word[i] = uint32_t((size_t(i) * g.block + off) / 2);
    g.sel[i] = (off & 1) ? 0x5432u : 0x3210u;
  }
  // a power of two d = 2^k divides 2^64: m = 2^(64 - k) exactly (k >= 1, so m fits 64 bits)
  g.mplane = (plane & (plane - 1)) == 0 ? (uint64_t(1) << 63) / uint64_t(plane) * 2 : spans_magic(uint64_t(plane));
  g.mnx = (p.nx & (p.nx - 1)) == 0 ? (uint64_t(1) << 63) / uint64_t(p.nx) * 2 : spans_magic(uint64_t(p.nx));
  return g;
}

inline size_t spans_smem_bytes(int stages, const SpansGeometry& g) { return 128 + size_t(stages) * g.stage_bytes; }

inline int spans_stages(const SpansGeometry& g, int ctas_per_sm) {
  const size_t budget = size_t(227 * 1024) / size_t(ctas_per_sm) - 1024;
  const size_t fit = (budget - 128) / g.stage_bytes;
  return fit >= 4 ? 4 : int(fit);
}

// Whether node (x, y, z) lies on a face whose nodes the face pass recomputes.
__device__ __forceinline__ bool on_pass_face(const StepPlan& p, int x, int y, int z) {
  const int m = p.face_mask;
  return ((m & 1) && x == 0) || ((m & 2) && x == p.nx - 1) || ((m & 4) && y == 0) || ((m & 8) && y == p.ny - 1) ||
         ((m & 16) && z == 0) || ((m & 32) && z == p.nz - 1);
}

template <typename S, int COLL, int STAGES, int WARPS, int MINB>
__global__ void __launch_bounds__(32 * (WARPS + 1), MINB)
    k_step_spans(const __grid_constant__ Planes<S> pl, const int8_t* __restrict__ flags, const __grid_constant__ StepPlan p,
                 const __grid_constant__ SpansGeometry g, int* __restrict__ err, long long wait_limit) {
  static_assert(is_16bit<S>(), "the span pipeline carries 16-bit storage");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + STAGES;
  unsigned char* stages = smem_raw + 128;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int TILE = spans_tile_nodes(WARPS);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], Q + 1);  // every producer lane that copies arrives with its own byte count
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
      unsigned char* st = stages + size_t(s) * g.stage_bytes;
      const int64_t t0 = int64_t(t) * TILE;
      if (lane < Q) {
        // [a, e): the sources of the tile widened to 8-element (16-byte) boundaries, clipped to
        // [0, ncell8); element a lands at the start of the block
        const int64_t src = t0 - g.d[lane];
        const int64_t a = src & ~int64_t(7);
        const int64_t e = (src + TILE + 7) & ~int64_t(7);
        const int64_t lo = a > 0 ? a : 0;
        const int64_t hi = e < g.ncell8 ? e : g.ncell8;
        if (hi > lo) {
          const unsigned bytes = unsigned(hi - lo) * unsigned(sizeof(S));
          mbar_arrive_expect_tx(&full[s], bytes);
          bulk_copy(reinterpret_cast<S*>(st) + size_t(lane) * g.block + (lo - a), pl.in[lane] + lo, bytes, &full[s]);
        } else {
          mbar_arrive(&full[s]);
        }
      } else if (lane == Q) {
        const int64_t hi = t0 + TILE < g.ncell16 ? t0 + TILE : g.ncell16;
        const unsigned bytes = unsigned(hi - t0);
        mbar_arrive_expect_tx(&full[s], bytes);
        bulk_copy(st + size_t(Q) * g.block * sizeof(S), flags + t0, bytes, &full[s]);
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
  const bool sr = p.rounding != 0;
  const uint32_t plane = uint32_t(p.nx) * uint32_t(p.ny);
  const uint32_t ncell = uint32_t(p.ncell);
  int k = 0;
  for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, k++) {
    const int s = k % STAGES;
    if (!mbar_wait(&full[s], (k / STAGES) & 1, wait_limit)) {
      if (ctid == 0) atomicExch(err, TMA_ERR_TIMEOUT);
      return;
    }
    const uint32_t* sw = reinterpret_cast<const uint32_t*>(stages + size_t(s) * g.stage_bytes) +
                         ROWS_NODES_PER_THREAD / 2 * ctid;  // two 16-bit values a word
    const int8_t* sflags = reinterpret_cast<const int8_t*>(stages + size_t(s) * g.stage_bytes) +
                           size_t(Q) * g.block * sizeof(S) + ROWS_NODES_PER_THREAD * ctid;
    const uint32_t n = uint32_t(t) * TILE + uint32_t(ROWS_NODES_PER_THREAD * ctid);
    const bool active = n < ncell;
    uint32_t fl4 = 0;
    uint32_t words[Q][2];
    int x = 0, y = 0, z = 0;
    bool interior = false;
    if (active) {
      z = int(__umul64hi(uint64_t(n), g.mplane));
      const uint32_t rem = n - uint32_t(z) * plane;
      y = int(__umul64hi(uint64_t(rem), g.mnx));
      x = int(rem - uint32_t(y) * uint32_t(p.nx));
      interior = x >= 1 && x + ROWS_NODES_PER_THREAD <= p.nx - 1 && y >= 1 && y <= p.ny - 2 && z >= 1 &&
                 z <= p.nz - 2;
      fl4 = *reinterpret_cast<const uint32_t*>(sflags);
      Unroll<0, Q>::run([&]<int I>() {
        const uint32_t* w = sw + g.word[I];
        const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
        words[I][0] = __byte_perm(w0, w1, g.sel[I]);
        words[I][1] = __byte_perm(w1, w2, g.sel[I]);
      });
    }
    // every value this warp reads from the stage is in registers: release it, so the producer
    // refills it while the collisions run rather than after them
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (!active) continue;
    if (!interior) {
      // a group at a face or across a row end: face nodes the face pass recomputes keep the staged
      // (meaningless) values; other face nodes gather theirs from global memory
      int live = 0;
      Unroll<0, ROWS_NODES_PER_THREAD>::run([&]<int J>() {
        int xj = x + J, yj = y, zj = z;
        if (xj >= p.nx) {
          xj -= p.nx;
          if (++yj == p.ny) {
            yj = 0;
            zj++;
          }
        }
        if (n + J >= ncell) return;
        const bool face = xj == 0 || xj == p.nx - 1 || yj == 0 || yj == p.ny - 1 || zj == 0 || zj == p.nz - 1;
        if (face && on_pass_face(p, xj, yj, zj)) return;
        live++;
        if (!face) return;
        S raw[Q];
        node_pull<S, false>(pl.in[0], flags, p, xj, yj, zj, int64_t(n) + J, raw);
        Unroll<0, Q>::run([&]<int I>() {
          const uint32_t b = uint32_t(PackedChunk<S, 2>::bits(raw[I]));
          uint32_t& w = words[I][J / 2];
          w = (J & 1) ? (w & 0x0000ffffu) | (b << 16) : (w & 0xffff0000u) | b;
        });
      });
      if (live == 0) continue;  // every node is left to the face pass or lies past the lattice
    }
    Unroll<0, 2>::run([&]<int J>() {
      const int8_t fa = int8_t(fl4 >> (16 * J)), fb = int8_t(fl4 >> (16 * J + 8));
      float2 v[Q];
      Unroll<0, Q>::run([&]<int I>() { v[I] = unpack2<S>(words[I][J]); });
      pair_update<S, MODE_FUSED, COLL>(v, p, fa, fb);
      uint32_t h = 0, h2 = 0;
      if (sr) {
        h = node_hash(int64_t(n) + 2 * J, seed);
        h2 = second_hash(h);
      }
      pack_pair<S>(v, sr, h, h2, [&]<int I>(uint32_t w) { words[I][J] = w; });
    });
    if (n + ROWS_NODES_PER_THREAD <= ncell) {
      Unroll<0, Q>::run([&]<int I>() { *reinterpret_cast<uint2*>(pl.out[I] + n) = make_uint2(words[I][0], words[I][1]); });
    } else {  // the lattice's last group: only its nodes below ncell
      Unroll<0, Q>::run([&]<int I>() {
        unsigned short* o = reinterpret_cast<unsigned short*>(pl.out[I] + n);
        o[0] = (unsigned short)(words[I][0] & 0xffffu);
        if (n + 1 < ncell) o[1] = (unsigned short)(words[I][0] >> 16);
        if (n + 2 < ncell) o[2] = (unsigned short)(words[I][1] & 0xffffu);
      });
    }
  }
}

}  // namespace hlbm
