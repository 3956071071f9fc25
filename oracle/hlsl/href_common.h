// href_common.h -- TEST INFRASTRUCTURE ONLY: what every reference-module translation unit includes
// before it opens its namespace and includes the rewritten reference module (see gprt.h).
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GPRT_DEVICE 1

// threads for the per-pixel dispatch loops (0 = OpenMP's default)
inline int href_threads(int n) {
#ifdef _OPENMP
  return n > 0 ? n : omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
