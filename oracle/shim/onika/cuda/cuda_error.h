// Forwarding stand-in (test infrastructure only): see onika/math/basic_types.h.
#pragma once
#include <onika/math/basic_types.h>
