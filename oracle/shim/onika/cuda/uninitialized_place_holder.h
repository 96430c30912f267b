// Stand-in (test infrastructure only) for the placeholder type named in reduce.hpp.
#pragma once
#include <onika/math/basic_types.h>
namespace onika::cuda {
template <class T>
struct UnitializedPlaceHolder {
  T value;
  T& get_ref() { return value; }
};
}  // namespace onika::cuda
