// Test stand-in for the Onika math types a hippoLBM plugin's slots use (see ../scg/operator.h).
#pragma once
#include <cstddef>

namespace onika {
namespace math {
struct IJK {
  long i = 0, j = 0, k = 0;
};
struct Vec3d {
  double x = 0, y = 0, z = 0;
};
struct AABB {
  Vec3d bmin, bmax;
};
}  // namespace math
}  // namespace onika
