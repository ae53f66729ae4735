// Host-side helpers shared by the engine's translation units: thread-local
// error text and status propagation (the reference printed CUDA errors and
// carried on, include/util.hpp:14-20; here every failure becomes a status).
#pragma once

#include <cstdint>
#include <string>

#include "../../include/vine.h"

namespace vine {

void set_error(const std::string &msg);
inline int fail(int status, const std::string &msg) {
  set_error(msg);
  return status;
}

}  // namespace vine

// Evaluates a CUDA runtime call; on failure records the error and returns
// VINE_ERR_CUDA from the enclosing function.
#define VINE_CUDA_TRY(expr)                                                         \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess)                                                          \
      return vine::fail(VINE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define VINE_TRY(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != VINE_OK) return _s; \
  } while (0)
