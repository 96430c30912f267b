// Stand-in (test infrastructure only) for Onika's 4x4 matrix and quadric evaluation, which
// are not part of the reference tree.  quadric_eval is this project's restatement:
// p^T Q p with p = (x, y, z, 1), accumulated row by row; quadric parity is therefore
// unpinned by the reference.
#pragma once
#include <onika/math/basic_types.h>
namespace onika::math {
struct Mat4d {
  double m[4][4];
};
inline double quadric_eval(const Mat4d& q, const Vec3d& v) {
  const double p[4] = {v.x, v.y, v.z, 1.0};
  double acc = 0.0;
  for (int i = 0; i < 4; i++) {
    double row = 0.0;
    for (int j = 0; j < 4; j++) row = row + q.m[i][j] * p[j];
    acc = acc + p[i] * row;
  }
  return acc;
}
}  // namespace onika::math
