// lanes.cuh -- arithmetic on one node (float, double) or on two nodes at once (float2), with
// every operation explicit: no product is ever contracted into a fused multiply-add by the
// compiler, so a collision written once over these operations rounds identically whether a
// kernel runs it on one node or on a pair.
//
// The pair form maps to sm_100's packed FP32 instructions (add/sub/mul/fma .rn.f32x2): one
// instruction updates the same quantity of two nodes, which halves the arithmetic issue slots of
// the step kernels that carry node pairs (the 16-bit tiers store each direction of a pair as one
// packed word; the FP32 vectorised kernel loads one float2 per direction).  Each lane of a packed
// operation rounds exactly as the scalar operation on that lane's operands.
#pragma once
#include <cuda_runtime.h>

namespace hlbm {

template <typename V>
struct Lanes;

template <>
struct Lanes<float> {
  using S = float;  // the scalar type of one lane
  static constexpr int N = 1;
  static __device__ __forceinline__ float splat(float s) { return s; }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  // 1/a: the hardware approximation (rcp.approx, about 1 ulp) refined by one Newton-Raphson step
  // r + r (1 - a r); no branch and no call, identical in the pair form
  static __device__ __forceinline__ float rcp(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return __fmaf_rn(r, __fmaf_rn(-a, r, 1.0f), r);
  }
  static __device__ __forceinline__ float lane(float a, int) { return a; }
  // per-lane choice: t where take (bit k = lane k), else f
  static __device__ __forceinline__ float select(int take, float t, float f) { return (take & 1) ? t : f; }
};

template <>
struct Lanes<float2> {
  using S = float;
  static constexpr int N = 2;
  static __device__ __forceinline__ float2 splat(float s) { return make_float2(s, s); }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
  static __device__ __forceinline__ float2 sub(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
    return *reinterpret_cast<float2*>(&d);
  }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
  static __device__ __forceinline__ float2 rcp(float2 a) {
    float2 r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(a.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(a.y));
    return __ffma2_rn(r, __ffma2_rn(make_float2(-a.x, -a.y), r, make_float2(1.0f, 1.0f)), r);
  }
  static __device__ __forceinline__ float lane(float2 a, int k) { return k ? a.y : a.x; }
  static __device__ __forceinline__ float2 select(int take, float2 t, float2 f) {
    return make_float2((take & 1) ? t.x : f.x, (take & 2) ? t.y : f.y);
  }
};

template <>
struct Lanes<double> {
  using S = double;
  static constexpr int N = 1;
  static __device__ __forceinline__ double splat(double s) { return s; }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }
  static __device__ __forceinline__ double lane(double a, int) { return a; }
  static __device__ __forceinline__ double select(int take, double t, double f) { return (take & 1) ? t : f; }
};

}  // namespace hlbm
