// lbm_step_vec.cuh -- the fused step with NPT consecutive x-nodes per thread.
//
// Same step as k_step (lbm_step.cuh), for lattices without wall obstacles: every direction
// plane is read and written as one aligned vector per thread (16 bytes: double2, float4, 8 packed
// FP16/BF16 values; or 8 bytes at the highest occupancy target: float2, 4 packed 16-bit values),
// which multiplies the bytes each thread keeps in flight by NPT.  All loads
// of a thread are issued before the first shuffle consumes one, so they overlap.
// A pull along e_x = +-1 needs the neighbouring element of the next/previous thread's vector:
// it comes from a warp shuffle, and lanes at a warp edge fetch it with one scalar load (the
// element of the previous/next warp, or the periodic image / on-node bounce-back at a row
// end).  Warps never straddle rows: the x extent of a block is a multiple of 32 threads.
// The kernel applies no boundary operator: the launcher follows it with the face pass (k_faces),
// which recomputes the nodes of the faces those operators touch, so the per-node code here stays
// small.  The 4- and 2-byte tiers update the nodes in pairs, the two lanes of packed FP32
// arithmetic (lanes.cuh); the 16-bit tiers convert each pair into packed words.
#pragma once
#include <type_traits>

#include "lbm_step.cuh"

namespace hlbm {

// ------------------------------------------------------------------ vector chunks
template <typename S, int NPT>
struct Chunk;

// plain element arrays for 8- and 4-byte types
template <typename S, int NPT, typename V>
struct ArrayChunk {
  S e[NPT];
  __device__ __forceinline__ void load(const S* p) {
    const V v = __ldg(reinterpret_cast<const V*>(p));
    static_assert(sizeof(V) == sizeof(S) * NPT, "vector width");
    const S* s = reinterpret_cast<const S*>(&v);
#pragma unroll
    for (int k = 0; k < NPT; k++) e[k] = s[k];
  }
  __device__ __forceinline__ void store(S* p) const {
    V v;
    S* s = reinterpret_cast<S*>(&v);
#pragma unroll
    for (int k = 0; k < NPT; k++) s[k] = e[k];
    *reinterpret_cast<V*>(p) = v;
  }
  template <int K>
  __device__ __forceinline__ S get() const {
    return e[K];
  }
  template <int K>
  __device__ __forceinline__ void set(S v) {
    e[K] = v;
  }
  __device__ __forceinline__ S first() const { return e[0]; }
  __device__ __forceinline__ S last() const { return e[NPT - 1]; }
  // elements 2J and 2J + 1 as the two lanes of a pair
  template <int J>
  __device__ __forceinline__ float2 lanes() const {
    return make_float2(float(e[2 * J]), float(e[2 * J + 1]));
  }
  template <int J>
  __device__ __forceinline__ void set_lanes(float2 v) {
    e[2 * J] = S(v.x);
    e[2 * J + 1] = S(v.y);
  }
  // [prev, e0 .. e_{NPT-2}]
  __device__ __forceinline__ void shift_in_prev(S prev) {
#pragma unroll
    for (int k = NPT - 1; k > 0; k--) e[k] = e[k - 1];
    e[0] = prev;
  }
  // [e1 .. e_{NPT-1}, next]
  __device__ __forceinline__ void shift_in_next(S next) {
#pragma unroll
    for (int k = 0; k < NPT - 1; k++) e[k] = e[k + 1];
    e[NPT - 1] = next;
  }
};

template <>
struct Chunk<double, 2> : ArrayChunk<double, 2, double2> {};
template <>
struct Chunk<float, 4> : ArrayChunk<float, 4, float4> {};
template <>
struct Chunk<float, 2> : ArrayChunk<float, 2, float2> {};

// 16-bit types packed two per 32-bit word; element 2j is the low half of word j
template <typename S, int NPT>
struct PackedChunk {
  static constexpr int W = NPT / 2;
  unsigned w[W];
  __device__ __forceinline__ void load(const S* p) {
    if constexpr (W == 4) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
      w[0] = v.x;
      w[1] = v.y;
      w[2] = v.z;
      w[3] = v.w;
    } else {
      const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
      w[0] = v.x;
      w[1] = v.y;
    }
  }
  __device__ __forceinline__ void store(S* p) const {
    if constexpr (W == 4)
      *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    else
      *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
  }
  static __device__ __forceinline__ S as_s(unsigned short b) {
    S s;
    memcpy(&s, &b, 2);
    return s;
  }
  static __device__ __forceinline__ unsigned short bits(S s) {
    unsigned short b;
    memcpy(&b, &s, 2);
    return b;
  }
  template <int K>
  __device__ __forceinline__ S get() const {
    return as_s((unsigned short)((K & 1) ? (w[K / 2] >> 16) : (w[K / 2] & 0xffffu)));
  }
  template <int K>
  __device__ __forceinline__ void set(S v) {
    const unsigned b = bits(v);
    w[K / 2] = (K & 1) ? ((w[K / 2] & 0xffffu) | (b << 16)) : ((w[K / 2] & 0xffff0000u) | b);
  }
  // both elements of word J as the two lanes of a pair, in FP32 (the stored numbers: scaled
  // deviations)
  template <int J>
  __device__ __forceinline__ float2 lanes() const {
    if constexpr (std::is_same_v<S, __half>) {
      return __half22float2(*reinterpret_cast<const __half2*>(&w[J]));
    } else {
      return make_float2(__uint_as_float(w[J] << 16), __uint_as_float(w[J] & 0xffff0000u));
    }
  }
  __device__ __forceinline__ S first() const { return get<0>(); }
  __device__ __forceinline__ S last() const { return get<NPT - 1>(); }
  __device__ __forceinline__ void shift_in_prev(S prev) {
    // new word j = (old element 2j-1 low, old element 2j high)
#pragma unroll
    for (int j = W - 1; j > 0; j--) w[j] = __byte_perm(w[j - 1], w[j], 0x5432);
    w[0] = __byte_perm(unsigned(bits(prev)) << 16, w[0], 0x5432);
  }
  __device__ __forceinline__ void shift_in_next(S next) {
    // new word j = (old element 2j+1 low, old element 2j+2 high)
#pragma unroll
    for (int j = 0; j < W - 1; j++) w[j] = __byte_perm(w[j], w[j + 1], 0x5432);
    w[W - 1] = __byte_perm(w[W - 1], unsigned(bits(next)), 0x5432);
  }
};
template <>
struct Chunk<__half, 8> : PackedChunk<__half, 8> {};
template <>
struct Chunk<__half, 4> : PackedChunk<__half, 4> {};
template <>
struct Chunk<__nv_bfloat16, 8> : PackedChunk<__nv_bfloat16, 8> {};
template <>
struct Chunk<__nv_bfloat16, 4> : PackedChunk<__nv_bfloat16, 4> {};

template <typename S>
__device__ __forceinline__ S shfl_up1(S v) {
  if constexpr (sizeof(S) == 2) {
    unsigned short b;
    memcpy(&b, &v, 2);
    const unsigned r = __shfl_up_sync(0xffffffffu, unsigned(b), 1);
    const unsigned short rb = (unsigned short)r;
    S out;
    memcpy(&out, &rb, 2);
    return out;
  } else {
    return __shfl_up_sync(0xffffffffu, v, 1);
  }
}
template <typename S>
__device__ __forceinline__ S shfl_down1(S v) {
  if constexpr (sizeof(S) == 2) {
    unsigned short b;
    memcpy(&b, &v, 2);
    const unsigned r = __shfl_down_sync(0xffffffffu, unsigned(b), 1);
    const unsigned short rb = (unsigned short)r;
    S out;
    memcpy(&out, &rb, 2);
    return out;
  } else {
    return __shfl_down_sync(0xffffffffu, v, 1);
  }
}

template <int NPT>
__device__ __forceinline__ void load_flags(const int8_t* p, int8_t (&fl)[NPT]) {
  if constexpr (NPT == 8) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    const int8_t* b = reinterpret_cast<const int8_t*>(&v);
#pragma unroll
    for (int k = 0; k < 8; k++) fl[k] = b[k];
  } else if constexpr (NPT == 4) {
    const unsigned v = __ldg(reinterpret_cast<const unsigned*>(p));
#pragma unroll
    for (int k = 0; k < 4; k++) fl[k] = int8_t((v >> (8 * k)) & 0xff);
  } else {
    const unsigned short v = __ldg(reinterpret_cast<const unsigned short*>(p));
    fl[0] = int8_t(v & 0xff);
    fl[1] = int8_t(v >> 8);
  }
}

// ------------------------------------------------------------------ the kernel
// The direction planes of the two lattices, fin + I * stride and fout + I * stride, passed as
// kernel parameters: every thread addresses a plane as that constant plus its own 32-bit node
// offset, and holds no per-direction pointer in registers.
template <typename S>
struct Planes {
  const S* in[Q];
  S* out[Q];
};

template <typename S>
inline Planes<S> make_planes(const S* fin, S* fout, int64_t stride) {
  Planes<S> pl;
  for (int i = 0; i < Q; i++) {
    pl.in[i] = fin + i * stride;
    pl.out[i] = fout + i * stride;
  }
  return pl;
}

// Node offsets are 32-bit (nodes < 2^32: vec_eligible_bytes requires it).
template <typename S, typename R, bool STRICT, int MODE, int NPT, int COLL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_vec(const __grid_constant__ Planes<S> pl,
                                                     const int8_t* __restrict__ flags, const StepPlan p) {
  advance_seed<S, MODE>(p);
  const uint32_t seed = launch_seed<S>(p);
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;  // vector index along x
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const int nvec = p.nx / NPT;
  const bool valid = tx < nvec && y < p.ny;  // invalid lanes still take part in the shuffles
  const int lane = threadIdx.x & 31;
  const int x0 = tx < nvec ? tx * NPT : 0;
  const int yy = y < p.ny ? y : p.ny - 1;
  // a row on an operator face (y or z): the face pass computes all of it after this kernel.  The
  // condition is uniform over the warp (one row), so no shuffle partner is missing.
  if (MODE != MODE_PROLOGUE && (p.face_mask >> 2) != 0 &&
      (((p.face_mask >> 2) & 1) && yy == 0 || ((p.face_mask >> 3) & 1) && yy == p.ny - 1 ||
       ((p.face_mask >> 4) & 1) && z == 0 || ((p.face_mask >> 5) & 1) && z == p.nz - 1))
    return;
  const uint32_t row = (uint32_t(z) * uint32_t(p.ny) + uint32_t(yy)) * uint32_t(p.nx);
  const uint32_t own = row + uint32_t(x0);
  Chunk<S, NPT> c[Q];
  if (MODE == MODE_PROLOGUE) {
    Unroll<0, Q>::run([&]<int I>() { c[I].load(pl.in[I] + own); });
  } else {
    // source row offsets for the y and z components (k = 1 - e): periodic axes wrap, others mark
    // the row "outside" (every node of the vector then bounces back on itself)
    uint32_t srow[3][3];
    bool out[3][3];
    {
      int sy[3], sz[3];
      bool oy[3], oz[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int d = 1 - k;
        int cy = yy - d, cz = z - d;
        oy[k] = oz[k] = false;
        if (cy < 0 || cy >= p.ny) {
          if (p.periodic[1]) cy = cy < 0 ? cy + p.ny : cy - p.ny; else oy[k] = true;
        }
        if (cz < 0 || cz >= p.nz) {
          if (p.periodic[2]) cz = cz < 0 ? cz + p.nz : cz - p.nz; else oz[k] = true;
        }
        sy[k] = cy;
        sz[k] = cz;
      }
#pragma unroll
      for (int ky = 0; ky < 3; ky++)
#pragma unroll
        for (int kz = 0; kz < 3; kz++) {
          srow[ky][kz] = (uint32_t(sz[kz]) * uint32_t(p.ny) + uint32_t(sy[ky])) * uint32_t(p.nx);
          out[ky][kz] = oy[ky] || oz[kz];
        }
    }
    // phase 1: issue every load (vectors, and the scalar edge elements of lanes at a warp or
    // row edge) before any of them is consumed, so that they are all in flight together
    const bool row_end = x0 + NPT >= p.nx;
    const bool left_lane = lane == 0 && valid, right_lane = (lane == 31 || row_end) && valid;
    S edge[Q];
    Unroll<0, Q>::run([&]<int I>() {
      constexpr int ex = D3Q19::ex[I], ky = 1 - D3Q19::ey[I], kz = 1 - D3Q19::ez[I];
      constexpr int O = D3Q19::opp(I);
      const S* plane = pl.in[I];
      const S* oplane = pl.in[O];
      if (out[ky][kz]) {  // uniform over the warp
        c[I].load(oplane + own);
        return;
      }
      const uint32_t src = srow[ky][kz];
      c[I].load(plane + src + uint32_t(x0));
      if constexpr (ex == 1) {  // node 0 pulls from x0 - 1
        if (left_lane)
          edge[I] = x0 > 0 ? ld_stream(plane + src + uint32_t(x0 - 1))
                           : (p.periodic[0] ? ld_stream(plane + src + uint32_t(p.nx - 1)) : ld_stream(oplane + own));
      } else if constexpr (ex == -1) {  // node NPT-1 pulls from x0 + NPT
        if (right_lane)
          edge[I] = !row_end ? ld_stream(plane + src + uint32_t(x0 + NPT))
                             : (p.periodic[0] ? ld_stream(plane + src) : ld_stream(oplane + own + uint32_t(NPT - 1)));
      }
    });
    // phase 2: shift the x-pulled vectors by one node, taking the neighbour element from the
    // adjacent lane (or from the edge load)
    Unroll<0, Q>::run([&]<int I>() {
      constexpr int ex = D3Q19::ex[I], ky = 1 - D3Q19::ey[I], kz = 1 - D3Q19::ez[I];
      if constexpr (ex != 0) {
        if (out[ky][kz]) return;
        if constexpr (ex == 1) {
          S prev = shfl_up1<S>(c[I].last());
          if (lane == 0) prev = edge[I];
          c[I].shift_in_prev(prev);
        } else {
          S next = shfl_down1<S>(c[I].first());
          if (lane == 31 || row_end) next = edge[I];
          c[I].shift_in_next(next);
        }
      }
    });
  }
  if (!valid) return;
  int8_t fl[NPT];
  load_flags<NPT>(flags + own, fl);
  if constexpr (sizeof(S) < 8) {
    // node pairs (2j, 2j+1), updated in place in the vectors; the 16-bit tiers round a
    // direction's two results into one packed word
    const bool sr = MODE != MODE_FINISH && p.rounding;
    Unroll<0, NPT / 2>::run([&]<int J>() {
      constexpr int K0 = 2 * J;
      float2 v[Q];
      if constexpr (is_16bit<S>() && COLL != 0) {
        // MRT on the pair's two lanes (packed FP32 halves its arithmetic)
        Unroll<0, Q>::run([&]<int I>() { v[I] = c[I].template lanes<J>(); });
        pair_update<S, MODE, COLL>(v, p, fl[K0], fl[K0 + 1]);
      } else {
        // BGK, whose update is short, and the FP32 tier: one node at a time (fewer live registers)
        float a[Q], b[Q];
        Unroll<0, Q>::run([&]<int I>() {
          const float2 t = c[I].template lanes<J>();
          a[I] = t.x;
          b[I] = t.y;
        });
        if constexpr (MODE != MODE_FINISH) {
          if (fl[K0] == FLAG_FLUID) collide<float, false, COLL, is_16bit<S>()>(a, p);
          if (fl[K0 + 1] == FLAG_FLUID) collide<float, false, COLL, is_16bit<S>()>(b, p);
        }
        if (fl[K0] == FLAG_WALL)  // a wall node (scratch) stores the read-out value of a wall
          Unroll<0, Q>::run([&]<int I>() { a[I] = wall_value<S, I>(p); });
        if (fl[K0 + 1] == FLAG_WALL) Unroll<0, Q>::run([&]<int I>() { b[I] = wall_value<S, I>(p); });
        Unroll<0, Q>::run([&]<int I>() { v[I] = make_float2(a[I], b[I]); });
      }
      if constexpr (is_16bit<S>()) {
        uint32_t h = 0, h2 = 0;
        if (sr) {
          h = node_hash(int64_t(own) + K0, seed);
          h2 = second_hash(h);
        }
        pack_pair<S>(v, sr, h, h2, [&]<int I>(uint32_t w) { c[I].w[J] = w; });
      } else {
        Unroll<0, Q>::run([&]<int I>() { c[I].template set_lanes<J>(v[I]); });
      }
    });
  } else {
    Unroll<0, NPT>::run([&]<int K>() {
      const int x = x0 + K;
      R v[Q];
      Unroll<0, Q>::run([&]<int I>() { v[I] = load_value<S, R, I>(c[I].template get<K>(), p); });
      node_update<S, R, STRICT, MODE, COLL>(v, pl.in[0], int64_t(own) + K, x, yy, z, fl[K], p, false, false);
      store_node<S, R, MODE>(v, p, seed, int64_t(own) + K, [&]<int I>(S s) { c[I].template set<K>(s); });
    });
  }
  Unroll<0, Q>::run([&]<int I>() { c[I].store(pl.out[I] + own); });
}

}  // namespace hlbm
