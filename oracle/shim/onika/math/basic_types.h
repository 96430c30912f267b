// Minimal stand-in for the few Onika types and helpers that hippoLBM's kernel functor
// headers name (Vec3d, IJK, AABB, vector adaptors, parallel traits, YAML converters).
// TEST INFRASTRUCTURE ONLY: it lets oracle/ref_harness.cpp compile the reference's
// functor headers unchanged, from where they lie, so that the reference itself can pin
// the oracle.  Written for this purpose; it is not Onika's source.
#pragma once
#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <limits>
#include <span>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#ifndef ONIKA_HOST_DEVICE_FUNC
#define ONIKA_HOST_DEVICE_FUNC
#endif

namespace onika {
static std::ostream& lout = std::cout;

namespace math {
struct Vec3d {
  double x = 0, y = 0, z = 0;
};
inline Vec3d operator+(const Vec3d& a, const Vec3d& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3d operator-(const Vec3d& a, const Vec3d& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3d operator+(const Vec3d& a, double s) { return {a.x + s, a.y + s, a.z + s}; }
inline Vec3d operator-(const Vec3d& a, double s) { return {a.x - s, a.y - s, a.z - s}; }
inline Vec3d operator*(const Vec3d& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3d operator/(const Vec3d& a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline Vec3d& operator*=(Vec3d& a, double s) {
  a.x *= s;
  a.y *= s;
  a.z *= s;
  return a;
}
inline bool operator==(const Vec3d& a, const Vec3d& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
// dot/norm in x, y, z order
inline double dot(const Vec3d& a, const Vec3d& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(const Vec3d& a) { return std::sqrt(dot(a, a)); }
inline std::ostream& operator<<(std::ostream& os, const Vec3d& v) { return os << v.x << "," << v.y << "," << v.z; }

struct IJK {
  long i = 0, j = 0, k = 0;
};
inline std::ostream& operator<<(std::ostream& os, const IJK& v) { return os << v.i << "," << v.j << "," << v.k; }

struct AABB {
  Vec3d bmin, bmax;
};
}  // namespace math

namespace memory {
template <class T>
using CudaMMVector = std::vector<T>;
}

namespace cuda {
template <class T>
inline T* vector_data(std::vector<T>& v) {
  return v.data();
}
template <class T>
inline const T* vector_data(const std::vector<T>& v) {
  return v.data();
}
template <class T>
inline size_t vector_size(const std::vector<T>& v) {
  return v.size();
}
}  // namespace cuda

namespace parallel {
template <size_t N>
struct ParallelExecutionSpace {
  std::array<long, N> m_start;
  std::array<long, N> m_end;
};
template <class F>
struct ParallelForFunctorTraits {
  static inline constexpr bool RequiresBlockSynchronousCall = false;
  static inline constexpr bool CudaCompatible = false;
};
struct ParallelExecutionContext {};
struct ParallelExecutionWrapper {};
enum OmpScheduling { OMP_SCHED_STATIC = 0 };
struct ParallelForOptions {
  OmpScheduling omp_scheduling = OMP_SCHED_STATIC;
};
}  // namespace parallel
}  // namespace onika

struct onikaInt3_t {
  int x, y, z;
};

// The reference headers declare YAML converters for their box types; they are never
// called here, so a node that holds nothing is enough for them to compile.
namespace YAML {
struct Node {
  template <class T>
  void push_back(const T&) {}
  bool IsSequence() const { return false; }
  size_t size() const { return 0; }
  Node operator[](size_t) const { return Node{}; }
  template <class T>
  T as() const {
    return T{};
  }
};
template <class T>
struct convert;
}  // namespace YAML
