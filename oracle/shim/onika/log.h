// Forwarding stand-in (test infrastructure only).
#pragma once
#include <onika/math/basic_types.h>
