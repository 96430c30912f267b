// lbm_step.cuh -- the fused D3Q19 time-step kernel (one node per thread, pull scheme on
// two lattices, SoA populations over the real box, one flag byte per node).
//
// One launch advances the stored post-collision state C_k to C_{k+1}:
//
//   pull-stream from C_k  (periodic wrap by index arithmetic; on-node bounce-back where
//                          the source is outside a non-periodic face or is a wall)
//   -> post_stream_bcs / boundary_conditions  (node-local plane operators, deck order)
//   -> start_iteration set_distribution boxes
//   -> macro variables -> BGK or MRT collision  -> store C_{k+1}.
//
// This is the reference step (config_compute_loop.msp:27-37) re-phased: the reference keeps
// S_k = post-stream state and runs macro -> collide -> pre_stream_bcs -> streaming
// (step1, update_ghost, step2; streaming.cu:68-118) -> post_stream_bcs -> boundary_conditions.
// The swap streaming bounces populations back on the node when the neighbour is outside the
// ext box (streaming.hpp:62-64); wall_bounce_back (bounce_back.hpp:160-185) makes a fluid
// node's population pulled from a wall equal to its own post-collision opposite; the plane
// pre/post bounce-back pair (bounce_back.hpp:60-156) re-writes those same on-node values,
// plus the cavity_z_* increments (cavity.hpp:74-87).  All of them are node-local in a pull
// formulation, so they fuse.  MODE_PROLOGUE (collide S_0 in place of a pull) and MODE_FINISH
// (stream + BCs, no collision: yields S_k) complete the re-phasing.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "d3q19.cuh"
#include "lanes.cuh"

namespace hlbm {

enum StepMode : int { MODE_PROLOGUE = 0, MODE_FUSED = 1, MODE_FINISH = 2 };

// ------------------------------------------------------------------ 16-bit conversions
// Two FP32 values to one packed pair (hi in the upper 16 bits).  .rs is sm_100a's stochastic
// rounding: the discarded bits of each value get a random addend before truncation, from the
// low (lo) and high (hi) half-word of rbits (13 bits each for FP16, 16 for BF16); .rn rounds
// to nearest even.
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float hi, float lo, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float hi, float lo, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}
__device__ __forceinline__ uint32_t cvt_rn_f16x2(float hi, float lo) {
  uint32_t d;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
__device__ __forceinline__ uint32_t cvt_rn_bf16x2(float hi, float lo) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

// ------------------------------------------------------------------ storage codecs
// Populations are stored as S and computed in R.  Half-precision storage keeps the
// deviation (f_i - w_i * rho0) * scale, so that the stored numbers are small and their
// relative precision is spent on the part of f that varies.
template <typename S, typename R>
struct Codec;

template <>
struct Codec<double, double> {
  template <int I>
  __device__ static __forceinline__ double dec(double s, const StepPlan&) { return s; }
  template <int I>
  __device__ static __forceinline__ double enc(double v, const StepPlan&) { return v; }
};
template <>
struct Codec<float, float> {
  template <int I>
  __device__ static __forceinline__ float dec(float s, const StepPlan&) { return s; }
  template <int I>
  __device__ static __forceinline__ float enc(float v, const StepPlan&) { return v; }
};
// 16-bit types store d_i * scale, d_i = f_i - dref_i (dref: the storage reference of the plan).
// dec / enc convert full populations; decd / encd (and the stochastic encd_sr) convert the scaled
// deviations d_i * scale themselves, which the step kernels carry for these tiers.
template <>
struct Codec<__half, float> {
  template <int I>
  __device__ static __forceinline__ float decd(__half s, const StepPlan&) {
    return __half2float(s);
  }
  template <int I>
  __device__ static __forceinline__ __half encd(float d, const StepPlan&) {
    return __float2half_rn(d);
  }
  // stochastic rounding of a pair (lo, hi)
  template <int I>
  __device__ static __forceinline__ uint32_t encd_sr2(float lo, float hi, uint32_t r) {
    return cvt_rs_f16x2(hi, lo, r);
  }
  template <int I>
  __device__ static __forceinline__ uint32_t encd2(float lo, float hi) {
    return cvt_rn_f16x2(hi, lo);
  }
  template <int I>
  __device__ static __forceinline__ float dec(__half s, const StepPlan& p) {
    return fmaf(__half2float(s), (float)p.inv_scale, p.dref[I]);
  }
  template <int I>
  __device__ static __forceinline__ __half enc(float v, const StepPlan& p) {
    return encd<I>((v - p.dref[I]) * (float)p.scale, p);
  }
};
template <>
struct Codec<__nv_bfloat16, float> {
  template <int I>
  __device__ static __forceinline__ float decd(__nv_bfloat16 s, const StepPlan&) {
    return __bfloat162float(s);
  }
  template <int I>
  __device__ static __forceinline__ __nv_bfloat16 encd(float d, const StepPlan&) {
    return __float2bfloat16_rn(d);
  }
  template <int I>
  __device__ static __forceinline__ uint32_t encd_sr2(float lo, float hi, uint32_t r) {
    return cvt_rs_bf16x2(hi, lo, r);
  }
  template <int I>
  __device__ static __forceinline__ uint32_t encd2(float lo, float hi) {
    return cvt_rn_bf16x2(hi, lo);
  }
  template <int I>
  __device__ static __forceinline__ float dec(__nv_bfloat16 s, const StepPlan& p) {
    return fmaf(__bfloat162float(s), (float)p.inv_scale, p.dref[I]);
  }
  template <int I>
  __device__ static __forceinline__ __nv_bfloat16 enc(float v, const StepPlan& p) {
    return encd<I>((v - p.dref[I]) * (float)p.scale, p);
  }
};

template <typename S>
__device__ __forceinline__ S ld_stream(const S* p) {
  return __ldg(p);
}

// ------------------------------------------------------------------ storage rounding
// With 16-bit storage a round-to-nearest store loses every update smaller than half a storage
// quantum, so slowly evolving regions stagnate and the rounding error accumulates with one sign.
// Stochastic rounding rounds up with probability equal to the discarded fraction: unbiased.  The
// random bits are a hash of (node index, step number, direction) -- reproducible, and the same
// for a lattice stepped alone or inside a batch.
__device__ __forceinline__ uint32_t node_hash(int64_t idx, uint32_t seed) {
  uint32_t h = uint32_t(idx) * 0x9E3779B1u ^ (seed * 0x85EBCA77u + 0x165667B1u);
  h ^= h >> 16;  // integer finaliser (xor-shift / multiply rounds)
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}

// Random bits for the pair conversion of direction I from two independent hash words: one IMAD.
// The high half-word is the well-mixed top of h * K; the low half-word is a bijection of h's low
// bits plus h2's, so it is uniform and, between two directions, the offset is independent of the
// value it is added to.
__device__ __forceinline__ uint32_t second_hash(uint32_t h) {
  uint32_t g = (h ^ (h >> 15)) * 0x2C1B3C6Du;
  return g ^ (g >> 12);
}
template <int I>
__device__ __forceinline__ uint32_t pair_bits(uint32_t h, uint32_t h2) {
  constexpr uint32_t K = 0x9E3779B9u * (2u * I + 1u);
  return h * K + h2;
}

template <typename S>
constexpr bool is_16bit() {
  return sizeof(S) == 2;
}

// One value of a node pair rounded as the pair conversion rounds it: the pair of node idx is
// (idx & ~1, idx | 1), its random bits are pair_bits of the pair's first node, and the value takes
// the half-word of those bits its lane takes (low for the even node, high for the odd one).  Every
// kernel -- one node, two nodes or vectors per thread -- so rounds every value with the same
// random bits, and the stochastically rounded state does not depend on the kernel that stepped it.
template <typename S, int I>
__device__ __forceinline__ S encd_sr_lane(float d, int64_t idx, uint32_t h, uint32_t h2) {
  const uint32_t r = pair_bits<I>(h, h2);
  const bool odd = (idx & 1) != 0;
  const uint32_t w = Codec<S, float>::template encd_sr2<I>(odd ? 0.0f : d, odd ? d : 0.0f, r);
  const unsigned short b = (unsigned short)(odd ? (w >> 16) : (w & 0xffffu));
  S out;
  memcpy(&out, &b, 2);
  return out;
}

// ------------------------------------------------------------------ compile-time loops
template <int I, int N>
struct Unroll {
  template <class F>
  __device__ static __forceinline__ void run(F&& f) {
    f.template operator()<I>();
    Unroll<I + 1, N>::run(f);
  }
};
template <int N>
struct Unroll<N, N> {
  template <class F>
  __device__ static __forceinline__ void run(F&&) {}
};

// Stores the node's Q values to dst(I).  FP64 / FP32 tiers carry full populations; the 16-bit
// tiers carry deviations from the storage reference, rounded stochastically when the state is
// carried (MODE_PROLOGUE / MODE_FUSED with p.rounding; the bits of the node's pair,
// encd_sr_lane), else to nearest.  The branch is taken once per node: selecting per value would
// make the compiler evaluate both conversions.
template <typename S, typename R, int MODE, class Dst>
__device__ __forceinline__ void store_node(const R (&v)[Q], const StepPlan& p, uint32_t seed, int64_t idx, Dst&& dst) {
  if constexpr (is_16bit<S>()) {
    if (MODE != MODE_FINISH && p.rounding) {
      const uint32_t h = node_hash(idx & ~int64_t(1), seed);
      const uint32_t h2 = second_hash(h);
      Unroll<0, Q>::run([&]<int I>() { dst.template operator()<I>(encd_sr_lane<S, I>(float(v[I]), idx, h, h2)); });
    } else {
      Unroll<0, Q>::run([&]<int I>() { dst.template operator()<I>(Codec<S, R>::template encd<I>(v[I], p)); });
    }
  } else {
    Unroll<0, Q>::run([&]<int I>() { dst.template operator()<I>(Codec<S, R>::template enc<I>(v[I], p)); });
  }
}

// The launch's step number (the stochastic-rounding salt): from the plan, or from the device
// counter pair of a graph-replayed launch (see StepPlan::seed_dev).
template <typename S>
__device__ __forceinline__ uint32_t launch_seed(const StepPlan& p) {
  if constexpr (is_16bit<S>())
    if (p.seed_dev) return p.seed_dev[p.seed_parity];
  return p.seed;
}

// One thread of the grid moves the counter pair on: no block of this launch reads the other slot.
template <typename S, int MODE>
__device__ __forceinline__ void advance_seed(const StepPlan& p) {
  if constexpr (is_16bit<S>() && MODE != MODE_FINISH)
    if (p.seed_dev && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
      p.seed_dev[p.seed_parity ^ 1] = p.seed_dev[p.seed_parity] + 1u;
}

// A stored population as the step kernels carry it: the full value, or for the 16-bit tiers
// its scaled deviation from the storage reference (the stored number itself).  dref is symmetric (dref_i = dref_opp(i)), so an
// on-node bounce-back reads the opposite slot with the same meaning.
template <typename S, typename R, int I>
__device__ __forceinline__ R load_value(S raw, const StepPlan& p) {
  if constexpr (is_16bit<S>())
    return Codec<S, R>::template decd<I>(raw, p);
  else
    return Codec<S, R>::template dec<I>(raw, p);
}

template <typename R, int I>
__device__ __forceinline__ constexpr R weight() {
  return R(1.0) / R(D3Q19::wden[I]);
}

// The read-out value of a wall node (population 0) as the kernels carry it: 0, or for the 16-bit
// tiers the scaled deviation -dref_I * scale.
template <typename S, int I>
__device__ __forceinline__ float wall_value(const StepPlan& p) {
  if constexpr (is_16bit<S>())
    return -p.dref[I] * float(p.scale);
  else
    return 0.0f;
}

// The value a start_iteration set_distribution box writes into direction I (f_i = value * w_i,
// set_distribution.hpp:29-46), as the kernels carry it: full populations, or for the 16-bit tiers
// the scaled deviation from the storage reference.
template <typename S, typename R, int I>
__device__ __forceinline__ R set_value(double value, const StepPlan& p) {
  if constexpr (is_16bit<S>())
    return (__fmul_rn(R(value), weight<R, I>()) - R(p.dref[I])) * R(p.scale);
  else
    return R(value) * weight<R, I>();
}

// sum_{axis} e_axis * a_axis over the non-zero components in x, y, z order: the value of the
// reference's (ex * ax + ey * ay) + ez * az with integer ex (adding a signed zero leaves a
// non-zero sum unchanged).
template <int I, typename R>
__device__ __forceinline__ R edot(R ax, R ay, R az) {
  constexpr int cx = D3Q19::ex[I], cy = D3Q19::ey[I], cz = D3Q19::ez[I];
  R acc = R(0);
  bool first = true;
  if (cx != 0) {
    acc = cx > 0 ? ax : -ax;
    first = false;
  }
  if (cy != 0) {
    acc = first ? (cy > 0 ? ay : -ay) : (cy > 0 ? acc + ay : acc - ay);
    first = false;
  }
  if (cz != 0) {
    acc = first ? (cz > 0 ? az : -az) : (cz > 0 ? acc + az : acc - az);
  }
  return acc;
}

// ------------------------------------------------------------------ macro variables
// macro_variables.hpp:56-69: rho = sum f (index order, from 0), u = sum f e / rho when
// rho > 1e-14, no half-force shift.
template <typename R, bool STRICT>
__device__ __forceinline__ void macro(const R (&v)[Q], R& rho, R& ux, R& uy, R& uz) {
  rho = v[0];
#pragma unroll
  for (int i = 1; i < Q; i++) rho = rho + v[i];
  ux = ((((((((v[1] - v[2]) + v[7]) - v[8]) + v[9]) - v[10]) + v[11]) - v[12]) + v[13]) - v[14];
  uy = ((((((((v[3] - v[4]) + v[7]) - v[8]) - v[9]) + v[10]) + v[15]) - v[16]) + v[17]) - v[18];
  uz = ((((((((v[5] - v[6]) + v[11]) - v[12]) - v[13]) + v[14]) + v[15]) - v[16]) - v[17]) + v[18];
  if (rho > R(1.0e-14)) {
    if (STRICT) {
      ux = ux / rho;
      uy = uy / rho;
      uz = uz / rho;
    } else {
      const R inv = R(1) / rho;
      ux *= inv;
      uy *= inv;
      uz *= inv;
    }
  }
}

// ------------------------------------------------------------------ BGK (bgk.hpp:47-62)
template <typename R, bool STRICT>
__device__ __forceinline__ void bgk(R (&v)[Q], const StepPlan& p) {
  R rho, ux, uy, uz;
  macro<R, STRICT>(v, rho, ux, uy, uz);
  const R u_squ = (ux * ux + uy * uy + uz * uz);
  const R tau = R(p.tau), inv_tau = R(p.inv_tau);
  const R Fx = R(p.F[0]), Fy = R(p.F[1]), Fz = R(p.F[2]);
  const bool force = p.has_force != 0;
  Unroll<0, Q>::run([&]<int I>() {
    constexpr R w = weight<R, I>();
    const R eu = edot<I, R>(ux, uy, uz);
    const R feq = w * rho * (R(1.) + R(3.) * eu + R(4.5) * eu * eu - R(1.5) * u_squ);
    if (STRICT) {
      R d = (feq - v[I]) / tau;
      if (force) d = d + R(3.) * rho * w * edot<I, R>(Fx, Fy, Fz);
      v[I] = v[I] + d;
    } else {
      R d = (feq - v[I]) * inv_tau;
      if (force) d += R(3.) * rho * w * edot<I, R>(Fx, Fy, Fz);
      v[I] += d;
    }
  });
}

// ------------------------------------------------------------------ MRT (mrt.hpp:42-193)
// Moment basis rows, d'Humieres D3Q19 in the reference's order; each moment sums its
// populations in increasing index, the reference's term order.
struct MrtTables {
  static constexpr signed char M[19][19] = {
      {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
      {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
      {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
      {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
      {0, 0, 0, -4, 4, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
      {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
      {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
      {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
      {0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
      {0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
      {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1}};
  // back-transform coefficients num/den (mrt.hpp:129-173), moments in M's row order
  static constexpr short BN[19][19] = {
      {1, -5, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, 1, -1, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, -1, 1, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, 0, 0, 1, -1, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0, 0, 0},
      {1, -11, -1, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, 0, 0, 0, 0, 0, 0},
      {1, 4, 1, 1, 1, 1, 1, 0, 0, 1, 1, 1, 1, 1, 0, 0, 1, -1, 0},
      {1, 4, 1, -1, -1, -1, -1, 0, 0, 1, 1, 1, 1, 1, 0, 0, -1, 1, 0},
      {1, 4, 1, 1, 1, -1, -1, 0, 0, 1, 1, 1, 1, -1, 0, 0, 1, 1, 0},
      {1, 4, 1, -1, -1, 1, 1, 0, 0, 1, 1, 1, 1, -1, 0, 0, -1, -1, 0},
      {1, 4, 1, 1, 1, 0, 0, 1, 1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 1},
      {1, 4, 1, -1, -1, 0, 0, -1, -1, 1, 1, -1, -1, 0, 0, 1, 1, 0, -1},
      {1, 4, 1, 1, 1, 0, 0, -1, -1, 1, 1, -1, -1, 0, 0, -1, -1, 0, -1},
      {1, 4, 1, -1, -1, 0, 0, 1, 1, 1, 1, -1, -1, 0, 0, -1, 1, 0, 1},
      {1, 4, 1, 0, 0, 1, 1, 1, 1, -1, -1, 0, 0, 0, 1, 0, 0, 1, -1},
      {1, 4, 1, 0, 0, -1, -1, -1, -1, -1, -1, 0, 0, 0, 1, 0, 0, -1, 1},
      {1, 4, 1, 0, 0, 1, 1, -1, -1, -1, -1, 0, 0, 0, -1, 0, 0, 1, 1},
      {1, 4, 1, 0, 0, -1, -1, 1, 1, -1, -1, 0, 0, 0, -1, 0, 0, -1, -1}};
  // denominators by (row group, moment)
  static constexpr short BD_AXIS[19] = {19, 2394, 63, 10, 10, 10, 10, 10, 10, 18, 18, 12, 12, 1, 1, 1, 1, 1, 1};
  static constexpr short BD_DIAG[19] = {19, 1197, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8};
  static constexpr short BD_REST[19] = {19, 399, 21, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
};

template <int I>
__device__ __forceinline__ constexpr int mrt_den(int k) {
  return I == 0 ? MrtTables::BD_REST[k]
                : (I <= 6 ? (k == 9 || k == 10 ? (I <= 2 ? 18 : 36) : MrtTables::BD_AXIS[k])
                          : (k == 9 ? (I >= 15 ? 18 : 36) : (k == 10 ? (I >= 15 ? 36 : 72) : MrtTables::BD_DIAG[k])));
}

// DEVF: v holds scaled deviations from the storage reference (the MRT rest state, whose moments
// are rho0, e = -11 rho0, eps = w_eps rho0 and zero otherwise).  The moments of v are then the
// scaled deviations of the moments, the e / eps equilibria take the density deviation m[0], the
// quadratic equilibrium terms take one factor 1/scale, and the force term the full density.
template <typename R, bool STRICT, bool DEVF = false>
__device__ __forceinline__ void mrt(R (&v)[Q], const StepPlan& p) {
  R m[19];
  Unroll<0, 19>::run([&]<int K>() {
    R acc = R(0);
    bool first = true;
    Unroll<0, Q>::run([&]<int I>() {
      constexpr int c = MrtTables::M[K][I];
      if (c != 0) {
        const R term = (c == 1) ? v[I] : (c == -1 ? -v[I] : R(c) * v[I]);
        acc = first ? term : acc + term;
        first = false;
      }
    });
    m[K] = acc;
  });
  const R rho = m[0], e = m[1], eps = m[2], jx = m[3], qx = m[4], jy = m[5], qy = m[6], jz = m[7], qz = m[8],
          pxx3 = m[9], pixx3 = m[10], pww = m[11], piww = m[12], pxy = m[13], pyz = m[14], pxz = m[15],
          mx = m[16], my = m[17], mz = m[18];
  const R s9 = STRICT ? R(1) / R(p.tau) : R(p.inv_tau), s13 = s9;
  const R s1 = R(p.mrt[0]), s2 = R(p.mrt[1]), s4 = R(p.mrt[2]), s10 = R(p.mrt[3]), s16 = R(p.mrt[4]);
  const R weps = R(p.mrt[5]), wepsj = R(p.mrt[6]), wxx = R(p.mrt[7]);
  const R rho0 = R(1.);
  // DEVF: scaled deviation moments; a product of two scaled momenta carries one scale too many
  const R qs = DEVF ? R(p.inv_scale) : R(1);
  const R jxq = DEVF ? jx * qs : jx;
  const R jyq = DEVF ? jy * qs : jy;
  const R jx2 = jxq * jx, jy2 = jyq * jy, jz2 = (DEVF ? jz * qs : jz) * jz;
  const R jj = (jx2 + jy2 + jz2);
  // relaxation (mrt.hpp:103-126), rho0 = 1
  const R e_eq = R(-11) * rho + R(19) / rho0 * jj;
  const R eps_eq = weps * rho + wepsj / rho0 * jj;
  const R pxx3_eq = R(1) / (rho0) * (R(2) * jx2 - (jy2 + jz2));
  const R pww_eq = R(1) / rho0 * (jy2 - jz2);
  const R pxy_eq = R(1) / rho0 * jxq * jy;
  const R pyz_eq = R(1) / rho0 * jyq * jz;
  const R pxz_eq = R(1) / rho0 * jxq * jz;
  R mo[19];
  mo[0] = rho;
  mo[1] = e - s1 * (e - e_eq);
  mo[2] = eps - s2 * (eps - eps_eq);
  mo[3] = jx;
  mo[4] = qx - s4 * (qx + R(2.) / R(3.) * jx);
  mo[5] = jy;
  mo[6] = qy - s4 * (qy + R(2.) / R(3.) * jy);
  mo[7] = jz;
  mo[8] = qz - s4 * (qz + R(2.) / R(3.) * jz);
  mo[9] = pxx3 - s9 * (pxx3 - pxx3_eq);
  mo[10] = pixx3 - s10 * (pixx3 - wxx * pxx3_eq);
  mo[11] = pww - s9 * (pww - pww_eq);
  mo[12] = piww - s10 * (piww - wxx * pww_eq);
  mo[13] = pxy - s13 * (pxy - pxy_eq);
  mo[14] = pyz - s13 * (pyz - pyz_eq);
  mo[15] = pxz - s13 * (pxz - pxz_eq);
  mo[16] = mx - s16 * mx;
  mo[17] = my - s16 * my;
  mo[18] = mz - s16 * mz;
  // back-transform (mrt.hpp:129-173) then the force term (mrt.hpp:181-191)
  const bool force = p.has_force != 0;
  const R Fx = R(p.F[0]), Fy = R(p.F[1]), Fz = R(p.F[2]);
  Unroll<0, Q>::run([&]<int I>() {
    R acc = R(0);
    bool first = true;
    Unroll<0, 19>::run([&]<int K>() {
      constexpr int num = MrtTables::BN[I][K];
      if (num != 0) {
        constexpr R coef = R(num < 0 ? -num : num) / R(mrt_den<I>(K));
        const R term = coef * mo[K];
        if (first)
          acc = num < 0 ? -term : term;
        else
          acc = num < 0 ? acc - term : acc + term;
        first = false;
      }
    });
    if (force)
      acc = acc + R(3.) * (DEVF ? R(p.scale) * (R(p.rho0) + rho * qs) : rho) * weight<R, I>() * edot<I, R>(Fx, Fy, Fz);
    v[I] = acc;
  });
}

// Moments of the basis that are even (equal entries for opposite directions) or odd (opposite
// entries): rho, e, eps and the stress-like moments are even; momenta, heat fluxes and m_x,y,z odd.
constexpr bool mrt_even(int k) { return k <= 2 || (k >= 9 && k <= 15); }
constexpr bool mrt_conserved(int k) { return k == 0 || k == 3 || k == 5 || k == 7; }

// e_I . a for an odd direction I, whose first non-zero component is +1 (1, 3, 5, 7, 9, 11, 13,
// 15, 17): in x, y, z order with no negation.  Its opposite I + 1 has e . a = -(this) exactly.
template <int I, typename V>
__device__ __forceinline__ V edot_odd(V ax, V ay, V az) {
  using L = Lanes<V>;
  static_assert(I & 1, "odd directions only");
  constexpr int cx = D3Q19::ex[I], cy = D3Q19::ey[I], cz = D3Q19::ez[I];
  if constexpr (cx != 0) {
    static_assert(cx == 1, "first component +1");
    V acc = ax;
    if constexpr (cy != 0) acc = cy > 0 ? L::add(acc, ay) : L::sub(acc, ay);
    if constexpr (cz != 0) acc = cz > 0 ? L::add(acc, az) : L::sub(acc, az);
    return acc;
  } else if constexpr (cy != 0) {
    static_assert(cy == 1, "first component +1");
    V acc = ay;
    if constexpr (cz != 0) acc = cz > 0 ? L::add(acc, az) : L::sub(acc, az);
    return acc;
  } else {
    return az;
  }
}

// ------------------------------------------------------------------ packed 16-bit node pairs
// The two 16-bit values of a packed word as FP32 lanes (low half-word in .x).
template <typename S>
__device__ __forceinline__ float2 unpack2(uint32_t w) {
  if constexpr (sizeof(S) == 2 && std::is_same_v<S, __half>) {
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
  } else {
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
  }
}

// A node pair of a 16-bit tier in FP32 lanes, rounded into one packed word per direction: with
// stochastic rounding (sr) from the random bits pair_bits(h, h2) of the pair's first node, else to
// nearest.  dst(I, word) stores direction I.
template <typename S, class Dst>
__device__ __forceinline__ void pack_pair(const float2 (&v)[Q], bool sr, uint32_t h, uint32_t h2, Dst&& dst) {
  if (sr)
    Unroll<0, Q>::run([&]<int I>() {
      dst.template operator()<I>(Codec<S, float>::template encd_sr2<I>(v[I].x, v[I].y, pair_bits<I>(h, h2)));
    });
  else
    Unroll<0, Q>::run([&]<int I>() { dst.template operator()<I>(Codec<S, float>::template encd2<I>(v[I].x, v[I].y)); });
}

// ------------------------------------------------------------------ MRT, FMA tiers
// S_p = f_{2p-1} + f_{2p} and D_p = f_{2p-1} - f_{2p} for the nine opposite pairs p = 1..9.  The
// first pair with a non-zero coefficient in moment row K (0: the rest direction).
template <int K>
constexpr int mrt_first_term() {
  int first = 10;
  for (int P = 9; P >= 1; P--)
    if (MrtTables::M[K][2 * P - 1] != 0) first = P;
  return (mrt_even(K) && MrtTables::M[K][0] != 0) ? 0 : first;
}

// The MRT collision of every tier except strict FP64, in about half the reference's operations.
// Directions 2p-1 and 2p are opposites, so an even moment sums S_p and an odd one D_p (about half
// the terms of the full transform), and the back-transform (the exact inverse of the basis) gives
// each opposite pair from one even and one odd part E_p, O_p as E_p +- O_p.  Only the
// non-conserved moments change, so the update is f_i -= sum_k Minv[i][k] dm_k with
// dm_k = m_k - m_k*, the relaxation of moment k.  Same equilibria and rates as `mrt`; the
// operation order differs, so results agree with it to rounding.  V is one node (float, double)
// or a node pair (float2); every operation is explicit (Lanes), so the pair form rounds as the
// one-node form on each lane.
// DEVF: v holds scaled deviations from the storage reference (the MRT rest state, whose moments
// are rho0, e = -11 rho0, eps = w_eps rho0 and zero otherwise).  The moments of v are then the
// scaled deviations of the moments, the e / eps equilibria take the density deviation m[0], the
// quadratic equilibrium terms take one factor 1/scale, and the force term the full density.
template <typename V, bool DEVF>
__device__ __forceinline__ void mrt_fast(V (&v)[Q], const StepPlan& p) {
  using L = Lanes<V>;
  using T = typename L::S;
  // moments in each row's term order, from the pair parts S_p, D_p
  V m[19];
  auto term = [&]<int K, int P>(V x) {
    constexpr int c = P == 0 ? MrtTables::M[K][0] : MrtTables::M[K][2 * P - 1];
    if constexpr (c != 0) {
      if constexpr (mrt_first_term<K>() == P)
        m[K] = c == 1 ? x : L::mul(L::splat(T(c)), x);
      else
        m[K] = c == 1 ? L::add(m[K], x) : (c == -1 ? L::sub(m[K], x) : L::fma(L::splat(T(c)), x, m[K]));
    }
  };
  Unroll<0, 19>::run([&]<int K>() {
    if constexpr (mrt_even(K)) term.template operator()<K, 0>(v[0]);
  });
  {
    V S[10], D[10];
    Unroll<1, 10>::run([&]<int P>() {
      S[P] = L::add(v[2 * P - 1], v[2 * P]);
      D[P] = L::sub(v[2 * P - 1], v[2 * P]);
    });
    Unroll<0, 19>::run([&]<int K>() {
      Unroll<1, 10>::run([&]<int P>() { term.template operator()<K, P>(mrt_even(K) ? S[P] : D[P]); });
    });
  }
  const V rho = m[0], e = m[1], eps = m[2], jx = m[3], qx = m[4], jy = m[5], qy = m[6], jz = m[7], qz = m[8],
          pxx3 = m[9], pixx3 = m[10], pww = m[11], piww = m[12], pxy = m[13], pyz = m[14], pxz = m[15];
  const V s9 = L::splat(T(p.inv_tau)), s13 = s9;
  const V s1 = L::splat(T(p.mrt[0])), s2 = L::splat(T(p.mrt[1])), s4 = L::splat(T(p.mrt[2]));
  const V s10 = L::splat(T(p.mrt[3])), s16 = L::splat(T(p.mrt[4]));
  const V weps = L::splat(T(p.mrt[5])), wepsj = L::splat(T(p.mrt[6])), mwxx = L::splat(-T(p.mrt[7]));
  // DEVF: a product of two scaled momenta carries one scale too many
  const V qs = L::splat(DEVF ? T(p.inv_scale) : T(1));
  const V jxq = DEVF ? L::mul(jx, qs) : jx;
  const V jyq = DEVF ? L::mul(jy, qs) : jy;
  const V jzq = DEVF ? L::mul(jz, qs) : jz;
  const V jx2 = L::mul(jxq, jx), jy2 = L::mul(jyq, jy), jz2 = L::mul(jzq, jz);
  const V jj = L::add(L::add(jx2, jy2), jz2);
  const V e_eq = L::fma(L::splat(T(19)), jj, L::mul(L::splat(T(-11)), rho));
  const V eps_eq = L::fma(wepsj, jj, L::mul(weps, rho));
  const V pxx3_eq = L::sub(L::add(jx2, jx2), L::add(jy2, jz2));
  const V pww_eq = L::sub(jy2, jz2);
  const V two3 = L::splat(T(2) / T(3));
  V dm[19];
  dm[1] = L::mul(s1, L::sub(e, e_eq));
  dm[2] = L::mul(s2, L::sub(eps, eps_eq));
  dm[4] = L::mul(s4, L::fma(two3, jx, qx));
  dm[6] = L::mul(s4, L::fma(two3, jy, qy));
  dm[8] = L::mul(s4, L::fma(two3, jz, qz));
  dm[9] = L::mul(s9, L::sub(pxx3, pxx3_eq));
  dm[10] = L::mul(s10, L::fma(mwxx, pxx3_eq, pixx3));
  dm[11] = L::mul(s9, L::sub(pww, pww_eq));
  dm[12] = L::mul(s10, L::fma(mwxx, pww_eq, piww));
  dm[13] = L::mul(s13, L::sub(pxy, L::mul(jxq, jy)));
  dm[14] = L::mul(s13, L::sub(pyz, L::mul(jyq, jz)));
  dm[15] = L::mul(s13, L::sub(pxz, L::mul(jxq, jz)));
  dm[16] = L::mul(s16, m[16]);
  dm[17] = L::mul(s16, m[17]);
  dm[18] = L::mul(s16, m[18]);
  // back-transform of the changes: rest direction, then opposite pairs; + 3 rho w_i e_i.F with
  // the full density (3 w_i e_i.F from the plan)
  auto part = [&]<int I, bool WANT_EVEN>() {
    V acc{};
    bool first = true;
    Unroll<0, 19>::run([&]<int K>() {
      constexpr int num = MrtTables::BN[I][K];
      if constexpr (num != 0 && !mrt_conserved(K) && mrt_even(K) == WANT_EVEN) {
        constexpr T coef = T(num) / T(mrt_den<I>(K));
        acc = first ? L::mul(L::splat(coef), dm[K]) : L::fma(L::splat(coef), dm[K], acc);
        first = false;
      }
    });
    return acc;
  };
  v[0] = L::sub(v[0], part.template operator()<0, true>());
  Unroll<1, 10>::run([&]<int P>() {
    constexpr int A = 2 * P - 1, B = 2 * P;
    const V E = part.template operator()<A, true>();
    const V O = part.template operator()<A, false>();
    v[A] = L::sub(v[A], L::add(E, O));
    v[B] = L::sub(v[B], L::sub(E, O));
  });
  if (p.has_force != 0) {  // + 3 rho w_i e_i.F with the full density (3 w_i e_i.F from the plan)
    const V fr = DEVF ? L::mul(L::splat(T(p.scale)), L::fma(rho, qs, L::splat(T(p.rho0)))) : rho;
    Unroll<1, Q>::run([&]<int I>() {
      const T fw = sizeof(T) == 8 ? T(p.fw3[I]) : T(p.ffw3[I]);
      v[I] = L::fma(L::splat(fw), fr, v[I]);
    });
  }
}

// ------------------------------------------------------------------ Zou/He planes
// neumann_{x,y,z}_{0,l}<19> (neumann.hpp:27-258) as one table per face.
struct ZouHeFace {
  int axis, t1, t2, den_sign;
  int tang[9];
  int known[5];
  int A1[3], B1[3], A2[3], B2[3];
  int main_dst, main_src, main_sign;
  int diag[4][6];  // dst, src, s_n, s_t, t (1|2), sign of n_t
};
struct ZouHeTables {
  static constexpr ZouHeFace face[6] = {
      {0, 1, 2, -1, {3, 4, 5, 6, 15, 17, 18, 16, 0}, {2, 10, 8, 14, 12}, {3, 15, 17}, {4, 18, 16}, {5, 18, 15},
       {6, 17, 16}, 1, 2, 1, {{9, 10, 1, -1, 1, 1}, {7, 8, 1, 1, 1, -1}, {11, 12, 1, 1, 2, -1}, {13, 14, 1, -1, 2, 1}}},
      {0, 1, 2, 1, {3, 4, 5, 6, 15, 17, 18, 16, 0}, {1, 7, 9, 11, 13}, {3, 15, 17}, {4, 18, 16}, {5, 18, 15},
       {6, 17, 16}, 2, 1, -1,
       {{10, 9, -1, 1, 1, -1}, {8, 7, -1, -1, 1, 1}, {12, 11, -1, -1, 2, 1}, {14, 13, -1, 1, 2, -1}}},
      {1, 0, 2, -1, {1, 2, 5, 6, 11, 13, 14, 12, 0}, {4, 9, 8, 18, 16}, {1, 11, 13}, {2, 14, 12}, {5, 11, 14},
       {6, 13, 12}, 3, 4, 1, {{7, 8, 1, 1, 1, -1}, {10, 9, 1, -1, 1, 1}, {15, 16, 1, 1, 2, -1}, {17, 18, 1, -1, 2, 1}}},
      {1, 0, 2, 1, {1, 2, 5, 6, 11, 13, 14, 12, 0}, {3, 7, 10, 15, 17}, {1, 11, 13}, {2, 14, 12}, {5, 11, 14},
       {6, 13, 12}, 4, 3, -1,
       {{8, 7, -1, -1, 1, 1}, {9, 10, -1, 1, 1, -1}, {16, 15, -1, -1, 2, 1}, {18, 17, -1, 1, 2, -1}}},
      {2, 0, 1, -1, {0, 1, 2, 3, 4, 7, 9, 10, 8}, {6, 13, 12, 17, 16}, {1, 7, 9}, {2, 10, 8}, {3, 7, 10},
       {4, 9, 8}, 5, 6, 1, {{11, 12, 1, 1, 1, -1}, {14, 13, 1, -1, 1, 1}, {15, 16, 1, 1, 2, -1}, {18, 17, 1, -1, 2, 1}}},
      {2, 0, 1, 1, {0, 1, 2, 3, 4, 7, 9, 10, 8}, {5, 11, 14, 15, 18}, {1, 7, 9}, {2, 10, 8}, {3, 7, 10},
       {4, 9, 8}, 6, 5, -1,
       {{13, 14, -1, 1, 1, -1}, {12, 11, -1, -1, 1, 1}, {17, 18, -1, 1, 2, -1}, {16, 15, -1, -1, 2, 1}}}};
};

template <int F, typename R>
__device__ __forceinline__ void zouhe(R (&v)[Q], const double* U) {
  constexpr ZouHeFace z = ZouHeTables::face[F];
  const R un = R(U[z.axis]), ut1 = R(U[z.t1]), ut2 = R(U[z.t2]);
  R ts = v[z.tang[0]];
#pragma unroll
  for (int k = 1; k < 9; k++) ts = ts + v[z.tang[k]];
  R ks = v[z.known[0]];
#pragma unroll
  for (int k = 1; k < 5; k++) ks = ks + v[z.known[k]];
  const R den = z.den_sign > 0 ? (R(1.) + un) : (R(1.) - un);
  const R rho = (ts + R(2.) * ks) / den;
  const R n1 = (R(1.) / R(2.)) * ((v[z.A1[0]] + v[z.A1[1]] + v[z.A1[2]]) - (v[z.B1[0]] + v[z.B1[1]] + v[z.B1[2]])) -
               (R(1.) / R(3.)) * rho * ut1;
  const R n2 = (R(1.) / R(2.)) * ((v[z.A2[0]] + v[z.A2[1]] + v[z.A2[2]]) - (v[z.B2[0]] + v[z.B2[1]] + v[z.B2[2]])) -
               (R(1.) / R(3.)) * rho * ut2;
  const R mterm = (R(1.) / R(3.)) * rho * un;
  v[z.main_dst] = z.main_sign > 0 ? v[z.main_src] + mterm : v[z.main_src] - mterm;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const R ut = z.diag[k][4] == 1 ? ut1 : ut2;
    const R nt = z.diag[k][4] == 1 ? n1 : n2;
    const R a = z.diag[k][2] > 0 ? un : -un;
    const R comb = z.diag[k][3] > 0 ? a + ut : a - ut;
    const R val = v[z.diag[k][1]] + (R(1.) / R(6.)) * rho * comb;
    v[z.diag[k][0]] = z.diag[k][5] > 0 ? val + nt : val - nt;
  }
}

// lid_driven_cavity (lid_driven_cavity.hpp:49-61): f = feq(sum f, U)
template <typename R>
__device__ __forceinline__ void lid(R (&v)[Q], const double* U) {
  R rho = v[0];
#pragma unroll
  for (int i = 1; i < Q; i++) rho = rho + v[i];
  const R Ux = R(U[0]), Uy = R(U[1]), Uz = R(U[2]);
  const R u_squ = Ux * Ux + Uy * Uy + Uz * Uz;
  Unroll<0, Q>::run([&]<int I>() {
    const R eu = edot<I, R>(Ux, Uy, Uz);
    v[I] = weight<R, I>() * rho * (R(1.) + R(3.) * eu + R(4.5) * eu * eu - R(1.5) * u_squ);
  });
}

template <int F>
__device__ __forceinline__ bool on_face(int x, int y, int z, const StepPlan& p) {
  if (F == 0) return x == 0;
  if (F == 1) return x == p.nx - 1;
  if (F == 2) return y == 0;
  if (F == 3) return y == p.ny - 1;
  if (F == 4) return z == 0;
  return z == p.nz - 1;
}

// post_bounce_back over the non-periodic faces in launcher order x0, xl, y0, yl, z0, zl
// (post_bounce_back.cu:115-120): the value saved by pre_bounce_back is this node's own
// post-collision opposite population, plus the cavity increments of that face.
template <typename S, typename R>
__device__ __forceinline__ void post_bb(R (&v)[Q], const S* __restrict__ fin, int64_t idx, int x, int y, int z,
                                        const StepPlan& p) {
  Unroll<0, 6>::run([&]<int F>() {
    if (p.periodic[F / 2]) return;
    if (!on_face<F>(x, y, z, p)) return;
    Unroll<0, 5>::run([&]<int K>() {
      constexpr int dst = PlaneBB::post[F][K], src = PlaneBB::pre[F][K];
      R val = Codec<S, R>::template dec<src>(ld_stream(fin + src * p.stride + idx), p);
      for (int c = 0; c < p.ncav[F]; c++) val = val + R(p.cav[F][c][K]);
      v[dst] = val;
    });
  });
}

// The streamed (pulled) value of direction I at node (x, y, z): the post-collision population of
// the upstream node, or the node's own opposite one where the upstream node is outside a
// non-periodic face or (wall_bounce_back active) a wall.
template <typename S, typename R, int I>
__device__ __forceinline__ R pull_value(const S* __restrict__ fin, const int8_t* __restrict__ flags,
                                        const StepPlan& p, int x, int y, int z) {
  constexpr int O = D3Q19::opp(I);
  int sx = x - D3Q19::ex[I], sy = y - D3Q19::ey[I], sz = z - D3Q19::ez[I];
  bool out = false;
  if (sx < 0 || sx >= p.nx) { if (p.periodic[0]) sx = sx < 0 ? sx + p.nx : sx - p.nx; else out = true; }
  if (sy < 0 || sy >= p.ny) { if (p.periodic[1]) sy = sy < 0 ? sy + p.ny : sy - p.ny; else out = true; }
  if (sz < 0 || sz >= p.nz) { if (p.periodic[2]) sz = sz < 0 ? sz + p.nz : sz - p.nz; else out = true; }
  const int64_t self = ((int64_t)z * p.ny + y) * p.nx + x;
  const int64_t src = ((int64_t)sz * p.ny + sy) * p.nx + sx;
  if (!out && p.walls && I != 0 && flags[src] == FLAG_WALL) out = true;
  return out ? Codec<S, R>::template dec<O>(ld_stream(fin + O * p.stride + self), p)
             : Codec<S, R>::template dec<I>(ld_stream(fin + I * p.stride + src), p);
}

// zero_gradient (no reference counterpart): on face F the populations that enter from outside
// (the directions post_bounce_back restores) take the streamed values of the interior neighbour
// one node inside along the face normal.  It runs before the step as a pass over the face: a
// population I entering at a face node reaches the node by on-node bounce-back, i.e. from the
// node's own outgoing slot opp(I), which nothing else reads (its streaming target is outside the
// lattice).  The pass writes the neighbour's streamed value there, so the step kernels need no
// outlet code.  It reads only entering slots and interior nodes' slots, never the slots it
// writes.  (a, b) are the node's coordinates along the face's two other axes, in x, y, z order.
template <typename S, typename R, int F>
__device__ __forceinline__ void zero_gradient_node(S* __restrict__ fin, const int8_t* __restrict__ flags,
                                                   const StepPlan& p, int a, int b) {
  constexpr int axis = F / 2;
  const int c = (F & 1) ? (axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz)) - 1 : 0;
  const int m = (F & 1) ? c - 1 : c + 1;  // interior neighbour along the normal
  const int x = axis == 0 ? c : a, y = axis == 1 ? c : (axis == 0 ? a : b), z = axis == 2 ? c : b;
  const int64_t self = ((int64_t)z * p.ny + y) * p.nx + x;
  if (flags[self] != FLAG_FLUID) return;  // like the neumann / lid operators: fluid nodes only
  const int mx = axis == 0 ? m : x, my = axis == 1 ? m : y, mz = axis == 2 ? m : z;
  Unroll<0, 5>::run([&]<int K>() {
    constexpr int I = PlaneBB::post[F][K];
    constexpr int O = D3Q19::opp(I);
    const R v = pull_value<S, R, I>(fin, flags, p, mx, my, mz);
    fin[O * p.stride + self] = Codec<S, R>::template enc<O>(v, p);
  });
}

template <typename S, typename R>
__device__ __forceinline__ void plane_ops(R (&v)[Q], const S* __restrict__ fin, int64_t idx, int x, int y, int z,
                                          int8_t flag, const StepPlan& p) {
  for (int o = 0; o < p.nops; o++) {
    const PlaneOp& op = p.ops[o];
    if (op.kind == OP_POST_BB) {
      post_bb<S, R>(v, fin, idx, x, y, z, p);
      continue;
    }
    if (op.kind == OP_ZERO_GRADIENT) continue;  // applied by the outlet pass before the step
    if (flag != FLAG_FLUID) continue;  // neuman / lid functors act on fluid nodes only
    bool hit;
    switch (op.face) {
      case 0: hit = on_face<0>(x, y, z, p); break;
      case 1: hit = on_face<1>(x, y, z, p); break;
      case 2: hit = on_face<2>(x, y, z, p); break;
      case 3: hit = on_face<3>(x, y, z, p); break;
      case 4: hit = on_face<4>(x, y, z, p); break;
      default: hit = on_face<5>(x, y, z, p); break;
    }
    if (!hit) continue;
    if (op.kind == OP_LID) {
      lid<R>(v, op.u);
    } else {
      switch (op.face) {
        case 0: zouhe<0, R>(v, op.u); break;
        case 1: zouhe<1, R>(v, op.u); break;
        case 2: zouhe<2, R>(v, op.u); break;
        case 3: zouhe<3, R>(v, op.u); break;
        case 4: zouhe<4, R>(v, op.u); break;
        default: zouhe<5, R>(v, op.u); break;
      }
    }
  }
}

// ------------------------------------------------------------------ one node of the step
// BGK of every tier except FP64, over one node or a node pair.
// DEVF (16-bit storage): v holds scaled deviations v_i = scale * (f_i - w_i rho0) (w_i rho0 is the
// BGK storage reference): rho = rho0 + sum v / scale, u = (sum e v) / (scale rho), and per
// direction v_i <- (1 - 1/tau) v_i + (1/tau) w_i (sum v + scale rho P_i),
// P_i = e.u (3 + 4.5 e.u) - 1.5 u^2.  Every sum runs over small numbers, so FP32 keeps the
// deviations' own precision and its rounding does not accumulate into the mass the way a sum of
// full populations does.
// !DEVF (FP32 storage): v holds full populations; the same update with sum v = rho, scale = 1
// and rho0 = 0 is f_i <- (1 - 1/tau) f_i + (1/tau) feq_i, u = j / rho where rho > 1e-14
// (macro_variables.hpp:56-69), else u = j.
// feq_i / w_i - (sum v) = srho P_i is folded to two FMAs per direction: with eu = e_I.u for the
// odd direction I, g_I = base + eu (s3 + s45 eu) and g_{I+1} = base + eu (s45 eu - s3).
// The sums run over the opposite pairs: sum = v_0 + sum_p S_p and j_ax = sum_p e_{2p-1}[ax] D_p.
template <typename V, bool DEVF>
__device__ __forceinline__ void bgk_v(V (&v)[Q], const StepPlan& p) {
  using L = Lanes<V>;
  using T = typename L::S;
  // opposite-pair sums S_p = f_{2p-1} + f_{2p} and differences D_p = f_{2p-1} - f_{2p}, reduced as
  // balanced trees (depth 4 for the density, 3 for each momentum component) so the two lanes'
  // chains leave the scheduler independent work
  V S[10], D[10];
  Unroll<1, 10>::run([&]<int P>() {
    S[P] = L::add(v[2 * P - 1], v[2 * P]);
    D[P] = L::sub(v[2 * P - 1], v[2 * P]);
  });
  static_assert(D3Q19::ex[1] == 1 && D3Q19::ex[7] == 1 && D3Q19::ex[9] == 1 && D3Q19::ex[11] == 1 &&
                    D3Q19::ex[13] == 1 && D3Q19::ey[3] == 1 && D3Q19::ey[7] == 1 && D3Q19::ey[9] == -1 &&
                    D3Q19::ey[15] == 1 && D3Q19::ey[17] == 1 && D3Q19::ez[5] == 1 && D3Q19::ez[11] == 1 &&
                    D3Q19::ez[13] == -1 && D3Q19::ez[15] == 1 && D3Q19::ez[17] == -1,
                "momentum trees follow the D3Q19 direction order");
  const V sum = L::add(L::add(L::add(v[0], S[1]), L::add(S[2], S[3])),
                       L::add(L::add(L::add(S[4], S[5]), L::add(S[6], S[7])), L::add(S[8], S[9])));
  const V jx = L::add(L::add(L::add(D[1], D[4]), L::add(D[5], D[6])), D[7]);
  const V jy = L::sub(L::add(L::add(D[2], D[4]), L::add(D[8], D[9])), D[5]);
  const V jz = L::sub(L::add(L::add(D[3], D[6]), D[8]), L::add(D[7], D[9]));
  V srho, cu;
  if constexpr (DEVF) {
    const V rho = L::fma(sum, L::splat(T(p.inv_scale)), L::splat(T(p.rho0)));
    srho = L::mul(L::splat(T(p.scale)), rho);
    cu = L::rcp(srho);
  } else {
    srho = sum;
    V r = L::rcp(sum);
    Unroll<0, L::N>::run([&]<int K>() {  // macro_variables: no division at vanishing density
      if (!(L::lane(sum, K) > T(1.0e-14))) r = L::select(1 << K, L::splat(T(1)), r);
    });
    cu = r;
  }
  const V ux = L::mul(jx, cu), uy = L::mul(jy, cu), uz = L::mul(jz, cu);
  const V c15 = L::mul(L::splat(T(1.5)), L::fma(ux, ux, L::fma(uy, uy, L::mul(uz, uz))));
  const T om = T(p.inv_tau);
  const V om1 = L::splat(T(1) - om);
  const V base = L::fma(L::mul(L::splat(T(-1)), srho), c15, sum);
  const V s3 = L::mul(L::splat(T(3.)), srho), ms3 = L::mul(L::splat(T(-3.)), srho);
  const V s45 = L::mul(L::splat(T(4.5)), srho);
  v[0] = L::fma(L::splat(om * weight<T, 0>()), base, L::mul(om1, v[0]));
  Unroll<1, 10>::run([&]<int P>() {
    constexpr int I = 2 * P - 1;
    const V omw = L::splat(om * weight<T, I>());
    const V eu = edot_odd<I, V>(ux, uy, uz);
    const V gA = L::fma(eu, L::fma(eu, s45, s3), base);
    const V gB = L::fma(eu, L::fma(eu, s45, ms3), base);
    v[I] = L::fma(omw, gA, L::mul(om1, v[I]));
    v[I + 1] = L::fma(omw, gB, L::mul(om1, v[I + 1]));
  });
  if (p.has_force != 0)  // + 3 rho w_i e_i.F (bgk.hpp:58), 3 w_i e_i.F from the plan
    Unroll<1, Q>::run([&]<int I>() { v[I] = L::fma(L::splat(p.ffw3[I]), srho, v[I]); });
}

// The collision of a tier.  COLL: 0 BGK, 1 MRT, 2 chosen at run time
// by p.collision (mixed batches, read-out modes).  FP64 keeps the reference's BGK structure
// (strict: its operation order and divisions; otherwise FMA and reciprocal multiplies) and strict
// FP64 the reference's MRT; the other tiers run bgk_v / mrt_fast, on one node (V = R) or a node
// pair (V = float2).  DEV: the values are the scaled deviations of the 16-bit tiers.
template <typename R, bool STRICT, int COLL, bool DEV, typename V>
__device__ __forceinline__ void collide(V (&v)[Q], const StepPlan& p) {
  const bool use_bgk = COLL == 0 || (COLL == 2 && p.collision == 0);
  if constexpr (sizeof(R) == 8) {
    static_assert(sizeof(V) == 8, "FP64 collides one node at a time");
    if (use_bgk)
      bgk<R, STRICT>(v, p);
    else if constexpr (STRICT)
      mrt<R, true>(v, p);
    else
      mrt_fast<V, false>(v, p);
  } else {
    if (use_bgk)
      bgk_v<V, DEV>(v, p);
    else
      mrt_fast<V, DEV>(v, p);
  }
}

// Whether node (x, y, z) lies on a face whose boundary operators can change it (p.face_mask).
// Other boundary nodes skip the operator code: for the 16-bit tiers that also skips a conversion
// to full populations and back, which would round.
__device__ __forceinline__ bool on_op_face(const StepPlan& p, int x, int y, int z) {
  const int bits = int(x == 0) | int(x == p.nx - 1) << 1 | int(y == 0) << 2 | int(y == p.ny - 1) << 3 |
                   int(z == 0) << 4 | int(z == p.nz - 1) << 5;
  return (bits & p.face_mask) != 0;
}

// Whether the z-plane z is an operator face (a test that is uniform over a block of a z-plane).
__device__ __forceinline__ bool on_op_z_face(const StepPlan& p, int z) {
  return ((p.face_mask >> 4) & 1 && z == 0) || ((p.face_mask >> 5) & 1 && z == p.nz - 1);
}

// Everything after the gather: boundary operators on the nodes whose values were pulled
// (`pulled` false for a first step, which collides the initial state), start_iteration boxes,
// collision.  The 16-bit tiers carry scaled deviations; the boundary operators and the boxes work
// on full populations, so those nodes convert around them.
template <typename S, typename R, bool STRICT, int MODE, int COLL>
__device__ __forceinline__ void node_update(R (&v)[Q], const S* __restrict__ fin, int64_t idx, int x, int y, int z,
                                            int8_t flag, const StepPlan& p, bool pulled, bool edge) {
  constexpr bool DEV = is_16bit<S>();
  if (pulled && edge && p.nops > 0) {
    if constexpr (DEV) Unroll<0, Q>::run([&]<int I>() { v[I] = fmaf(v[I], R(p.inv_scale), R(p.dref[I])); });
    plane_ops<S, R>(v, fin, idx, x, y, z, flag, p);
    if constexpr (DEV) Unroll<0, Q>::run([&]<int I>() { v[I] = (v[I] - R(p.dref[I])) * R(p.scale); });
  }
  if (MODE != MODE_FINISH) {
    for (int s = 0; s < p.nsets; s++) {  // start_iteration: set_distribution boxes
      const SetBox& b = p.sets[s];
      if (x >= b.lo[0] && x <= b.hi[0] && y >= b.lo[1] && y <= b.hi[1] && z >= b.lo[2] && z <= b.hi[2])
        Unroll<0, Q>::run([&]<int I>() { v[I] = set_value<S, R, I>(b.value, p); });
    }
    if (flag == FLAG_FLUID) collide<R, STRICT, COLL, DEV>(v, p);
  }
}

// node_update for two nodes a and b of a 4- or 2-byte tier, the two lanes of v: a first step
// (MODE_PROLOGUE) or a fused step collides both lanes; a read-out (MODE_FINISH) leaves them.  The
// pair kernels take lattices whose non-fluid nodes are walls under wall_bounce_back
// (pair_kernels_apply): a wall node's populations are scratch that no fluid node reads, so it
// collides with its partner and then stores the read-out value of a wall.  No boundary operators
// (a face pass applies them) and no start_iteration boxes (plans with boxes run the one-node
// kernel).  Each fluid lane gets exactly the arithmetic node_update gives its node.
template <typename S, int MODE, int COLL>
__device__ __forceinline__ void pair_update(float2 (&v)[Q], const StepPlan& p, int8_t fa, int8_t fb) {
  constexpr bool DEV = is_16bit<S>();
  if constexpr (MODE != MODE_FINISH) collide<float, false, COLL, DEV>(v, p);
  const int wall = int(fa == FLAG_WALL) | int(fb == FLAG_WALL) << 1;
  if (wall)
    Unroll<0, Q>::run([&]<int I>() { v[I] = Lanes<float2>::select(wall, Lanes<float2>::splat(wall_value<S, I>(p)), v[I]); });
}

template <typename S, bool WALLS>
__device__ __forceinline__ void node_pull(const S* __restrict__ fin, const int8_t* __restrict__ flags,
                                          const StepPlan& p, int x, int y, int z, int64_t idx, S (&raw)[Q]);

// The stored values the node (x, y, z) gathers (pull with periodic wrap and on-node bounce-back;
// in the prologue its own values), every load issued before any is used.  A bounced value (the
// node's own opp(I) slot) decodes like a pulled one because the storage reference is symmetric.
template <typename S, int MODE, bool WALLS>
__device__ __forceinline__ void node_gather(const S* __restrict__ fin, const int8_t* __restrict__ flags,
                                            const StepPlan& p, int x, int y, int z, int64_t idx, S (&raw)[Q]) {
  if constexpr (MODE == MODE_PROLOGUE) {
    Unroll<0, Q>::run([&]<int I>() { raw[I] = ld_stream(fin + I * p.stride + idx); });
  } else {
    node_pull<S, WALLS>(fin, flags, p, x, y, z, idx, raw);
  }
}

// node_gather's pull: source coordinates x - e for e in {+1, 0, -1}; periodic axes wrap, others
// flag "outside" (on-node bounce-back), as do wall sources where wall_bounce_back is active.
template <typename S, bool WALLS>
__device__ __forceinline__ void node_pull(const S* __restrict__ fin, const int8_t* __restrict__ flags,
                                          const StepPlan& p, int x, int y, int z, int64_t idx, S (&raw)[Q]) {
  int sx[3], sy[3], sz[3];
  bool ox[3], oy[3], oz[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int d = 1 - k;  // component of e_i: +1, 0, -1 -> source offset -d
    int cx = x - d, cy = y - d, cz = z - d;
    ox[k] = oy[k] = oz[k] = false;
    if (cx < 0 || cx >= p.nx) {
      if (p.periodic[0]) cx = cx < 0 ? cx + p.nx : cx - p.nx; else ox[k] = true;
    }
    if (cy < 0 || cy >= p.ny) {
      if (p.periodic[1]) cy = cy < 0 ? cy + p.ny : cy - p.ny; else oy[k] = true;
    }
    if (cz < 0 || cz >= p.nz) {
      if (p.periodic[2]) cz = cz < 0 ? cz + p.nz : cz - p.nz; else oz[k] = true;
    }
    sx[k] = cx;
    sy[k] = cy;
    sz[k] = cz;
  }
  bool near = true;  // whether some pull may come from a wall node
  if constexpr (WALLS) near = p.nearwall == nullptr || p.nearwall[idx] != 0;
  Unroll<0, Q>::run([&]<int I>() {
    constexpr int kx = 1 - D3Q19::ex[I], ky = 1 - D3Q19::ey[I], kz = 1 - D3Q19::ez[I];
    constexpr int O = D3Q19::opp(I);
    bool bounce = ox[kx] || oy[ky] || oz[kz];
    const int64_t src = ((int64_t)sz[kz] * p.ny + sy[ky]) * p.nx + sx[kx];
    if (WALLS && I != 0 && !bounce && near) bounce = (flags[src] == FLAG_WALL);
    raw[I] = ld_stream(bounce ? fin + O * p.stride + idx : fin + I * p.stride + src);
  });
}

// The whole step for the node (x, y, z): gather, boundary operators (unless OPS is false: a face
// pass applies them), start_iteration boxes, collision, store.
template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int COLL, bool OPS = true>
__device__ __forceinline__ void node_step(const S* __restrict__ fin, S* __restrict__ fout,
                                          const int8_t* __restrict__ flags, const StepPlan& p, int x, int y, int z) {
  const int64_t idx = ((int64_t)z * p.ny + y) * p.nx + x;
  const int8_t flag = flags[idx];
  if (WALLS && flag == FLAG_WALL) {
    if (MODE == MODE_FINISH)
      Unroll<0, Q>::run([&]<int I>() { fout[I * p.stride + idx] = Codec<S, R>::template enc<I>(R(0), p); });
    return;
  }
  S raw[Q];
  node_gather<S, MODE, WALLS>(fin, flags, p, x, y, z, idx, raw);
  R v[Q];
  Unroll<0, Q>::run([&]<int I>() { v[I] = load_value<S, R, I>(raw[I], p); });
  node_update<S, R, STRICT, MODE, COLL>(v, fin, idx, x, y, z, flag, p, MODE != MODE_PROLOGUE,
                                        OPS && on_op_face(p, x, y, z));
  store_node<S, R, MODE>(v, p, launch_seed<S>(p), idx, [&]<int I>(S s) { fout[I * p.stride + idx] = s; });
}

// Storage types whose one-node step kernel leaves the boundary operators to the face pass (k_faces):
// the 4- and 2-byte tiers, whose kernels are bound by instruction issue, so the operator code
// costs there.  FP64 applies them inline: its kernel runs at the copy bandwidth either way.
template <typename S>
constexpr bool face_pass_tier() {
  return sizeof(S) < 8;
}

// ------------------------------------------------------------------ the step kernel
template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int COLL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step(const S* __restrict__ fin, S* __restrict__ fout,
                                                    const int8_t* __restrict__ flags, const StepPlan p) {
  advance_seed<S, MODE>(p);
  int x, y, z;
  if (p.linear) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.nx * p.ny) return;
    z = blockIdx.y;
    y = __float2int_rz(float(i) * p.inv_nx);  // i / nx within one (exact below 2^24, see StepPlan)
    x = i - y * p.nx;
    if (x < 0) {
      y--;
      x += p.nx;
    } else if (x >= p.nx) {
      y++;
      x -= p.nx;
    }
  } else {
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z = blockIdx.z;
    if (x >= p.nx || y >= p.ny) return;
  }
  // the face pass computes the operator faces after this kernel (not after a prologue): whole
  // z-face planes are skipped (a uniform test per block), other face nodes are computed twice
  if (face_pass_tier<S>() && MODE != MODE_PROLOGUE && on_op_z_face(p, z)) return;
  node_step<S, R, STRICT, MODE, WALLS, COLL, !face_pass_tier<S>()>(fin, fout, flags, p, x, y, z);
}

// The one-node step of the 16-bit tiers, two consecutive nodes of a z-plane per thread: each
// direction's two results convert into one packed word and one 32-bit store (plane sizes even, so
// every pair starts on a 4-byte boundary; below 2^24 nodes, for the index arithmetic of `linear`).
// Boundary operators are left to the face pass.  A wall node of a pair stores the read-out value
// of a wall (population 0); the one-node kernel leaves that slot untouched, and no fluid node
// reads it either way.
template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int COLL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_pairs(const S* __restrict__ fin, S* __restrict__ fout,
                                                          const int8_t* __restrict__ flags, const StepPlan p) {
  static_assert(is_16bit<S>(), "packed pairs are 16-bit storage");
  advance_seed<S, MODE>(p);
  const int plane = p.nx * p.ny;
  const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= plane) return;
  const int z = blockIdx.y;
  int y = __float2int_rz(float(i) * p.inv_nx);  // i / nx, exact after one correction below 2^24
  int x = i - y * p.nx;
  if (x < 0) {
    y--;
    x += p.nx;
  } else if (x >= p.nx) {
    y++;
    x -= p.nx;
  }
  int xb = x + 1, yb = y;
  if (xb == p.nx) {
    xb = 0;
    yb++;
  }
  // a z-face plane: the face pass computes it after this kernel
  if (MODE != MODE_PROLOGUE && on_op_z_face(p, z)) return;
  const int64_t idx = int64_t(z) * plane + i;
  const int8_t fa = flags[idx], fb = flags[idx + 1];
  S ra[Q], rb[Q];
  node_gather<S, MODE, WALLS>(fin, flags, p, x, y, z, idx, ra);
  node_gather<S, MODE, WALLS>(fin, flags, p, xb, yb, z, idx + 1, rb);
  float2 v[Q];  // node a in .x, node b in .y
  Unroll<0, Q>::run([&]<int I>() { v[I] = make_float2(load_value<S, R, I>(ra[I], p), load_value<S, R, I>(rb[I], p)); });
  pair_update<S, MODE, COLL>(v, p, fa, fb);
  const bool sr = MODE != MODE_FINISH && p.rounding;
  uint32_t h = 0, h2 = 0;
  if (sr) {
    h = node_hash(idx, launch_seed<S>(p));
    h2 = second_hash(h);
  }
  pack_pair<S>(v, sr, h, h2, [&]<int I>(uint32_t w) { *reinterpret_cast<uint32_t*>(fout + I * p.stride + idx) = w; });
}

// The face pass of the vectorised kernels: the nodes of the faces in `faces` (bit F = face F),
// each stepped whole by node_step, after the vectorised kernel stepped them without boundary
// operators.  Both read only fin, so the pass overwrites those nodes' outputs with the complete
// update.  blockIdx.y is the face; nodes on two faces are computed twice, to the same bits.
template <typename S, typename R, bool STRICT, int MODE, bool WALLS, int COLL>
__global__ void __launch_bounds__(256) k_faces(const S* __restrict__ fin, S* __restrict__ fout,
                                               const int8_t* __restrict__ flags, const StepPlan p, int faces) {
  const int F = blockIdx.y;
  if (!(faces >> F & 1)) return;
  if ((faces & 3) == 3 && F < 2) {
    // both x faces in one interleaved sweep: thread i takes x = nx - 1 of row (i + 1) / 2 for even i
    // and x = 0 of that row for odd i (row 0's x = 0 last), so neighbouring threads step nodes
    // that are neighbours in memory (the end of one row, the start of the next) and share the
    // sectors of their loads and stores; the two faces' nodes alone lie nx elements apart
    if (F == 1) return;
    const int64_t rows = int64_t(p.ny) * p.nz;
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= 2 * rows) return;
    int64_t r = (i + 1) >> 1;
    const int x = ((i + 1) & 1) ? p.nx - 1 : 0;
    if (r == rows) r = 0;
    const int z = int(r / p.ny), y = int(r - int64_t(z) * p.ny);
    node_step<S, R, STRICT, MODE, WALLS, COLL>(fin, fout, flags, p, x, y, z);
    return;
  }
  const int axis = F / 2;
  const int na = axis == 0 ? p.ny : p.nx;  // the face's two axes, in x, y, z order
  const int nb = axis == 2 ? p.ny : p.nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na * nb) return;
  const int a = i % na, b = i / na;
  const int c = (F & 1) ? (axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz)) - 1 : 0;
  const int x = axis == 0 ? c : a;
  const int y = axis == 1 ? c : (axis == 0 ? a : b);
  const int z = axis == 2 ? c : b;
  node_step<S, R, STRICT, MODE, WALLS, COLL>(fin, fout, flags, p, x, y, z);
}

// The wall fix-up after the vectorised kernel, which pulls without testing for wall nodes: every
// node the near-wall map marks (some pull may come from a wall) is stepped again by the one-node
// step with the wall test, and a read-out gives wall nodes the read-out value of a wall.  It runs
// after the face pass and reads only fin, so its result replaces both.
template <typename S, typename R, bool STRICT, int MODE, int COLL>
__global__ void __launch_bounds__(256) k_wall_fixup(const S* __restrict__ fin, S* __restrict__ fout,
                                                    const int8_t* __restrict__ flags, const StepPlan p) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= p.ncell) return;
  const bool near = p.nearwall == nullptr || p.nearwall[idx] != 0;
  if (!near && !(MODE == MODE_FINISH && flags[idx] == FLAG_WALL)) return;
  const int64_t plane = int64_t(p.nx) * p.ny;
  const int z = int(idx / plane);
  const int64_t r = idx - int64_t(z) * plane;
  const int y = int(r / p.nx), x = int(r - int64_t(y) * p.nx);
  node_step<S, R, STRICT, MODE, true, COLL>(fin, fout, flags, p, x, y, z);
}

}  // namespace hlbm
