// Test stand-in for onika::fatal_error (see scg/operator.h): the message, then an exception.
#pragma once
#include <sstream>
#include <stdexcept>
#include <string>

namespace onika {
struct FatalError {
  std::ostringstream os;
  template <class T>
  FatalError& operator<<(const T& v) {
    os << v;
    return *this;
  }
  FatalError& operator<<(std::ostream& (*)(std::ostream&)) { throw std::runtime_error(os.str()); }
};
inline FatalError fatal_error() { return {}; }
}  // namespace onika
