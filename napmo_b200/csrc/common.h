// Shared definitions for the napmo_b200 native library: status codes, the
// thread-local last-error slot that every C-ABI entry point reports through,
// and CUDA error checking.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace napmo {

// Status codes returned by every int-returning C-ABI entry point.
constexpr int kOk = 0;
constexpr int kInvalidArgument = 1;
constexpr int kCudaError = 2;
constexpr int kOutOfMemory = 3;
constexpr int kNotSupported = 4;
constexpr int kDeviceTimeout = 5;

// Records an error for napmo_last_error(); returns the code so call sites can
// `return set_error(...)`.
int set_error(int code, const std::string &msg);
void clear_error();

}  // namespace napmo

#ifdef __CUDACC__
#define NAPMO_CUDA_TRY(expr)                                                   \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      return ::napmo::set_error(::napmo::kCudaError,                           \
                                std::string(#expr ": ") +                      \
                                    cudaGetErrorString(_e));                   \
    }                                                                          \
  } while (0)
#endif

#define NAPMO_REQUIRE(cond, msg)                                               \
  do {                                                                         \
    if (!(cond)) {                                                             \
      return ::napmo::set_error(::napmo::kInvalidArgument, (msg));             \
    }                                                                          \
  } while (0)
