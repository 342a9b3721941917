// Internal host-side definitions shared by the library's translation units.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "coffee_b200.h"

namespace coffee {

// Record a failure for coffee_last_error_string() and return `code`.
int fail(int code, const char* fmt, ...);
void clear_error();

}  // namespace coffee

#define COFFEE_CUDA_TRY(call)                                                         \
  do {                                                                                \
    cudaError_t err__ = (call);                                                       \
    if (err__ != cudaSuccess)                                                         \
      return coffee::fail(err__ == cudaErrorMemoryAllocation ? COFFEE_E_NOMEM          \
                                                             : COFFEE_E_CUDA,         \
                          "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err__),   \
                          __FILE__, __LINE__);                                        \
  } while (0)
