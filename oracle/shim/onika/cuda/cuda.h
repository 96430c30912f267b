// Stand-in for the Onika CUDA portability macros the reference's reduction functor names
// (test infrastructure only).  The oracle harness runs those functors serially on the host,
// so the "atomics" are plain read-modify-writes.
#pragma once
#include <onika/math/basic_types.h>
#define ONIKA_CU_ATOMIC_ADD(a, b) ((a) += (b))
#define ONIKA_CU_ATOMIC_MIN(a, b) ((a) = std::min((a), (b)))
#define ONIKA_CU_ATOMIC_MAX(a, b) ((a) = std::max((a), (b)))
#define ONIKA_CU_BLOCK_SHARED static
#define ONIKA_CU_THREAD_IDX 0
#define ONIKA_CU_BLOCK_SYNC() \
  do {                        \
  } while (0)
#define ONIKA_CU_DEVICE_SYNCHRONIZE() \
  do {                                \
  } while (0)
