// see operator.h (test stand-in for Onika)
#pragma once
#include "operator.h"
