// Helpers shared by the C-ABI translation units: device buffers, the
// library stream used by the host-pointer (nAPMO-compatible) entry points,
// and exception-to-status conversion.
#pragma once

#include <cuda_runtime.h>

#include <exception>
#include <string>
#include <vector>

#include "common.h"

namespace napmo {

// Stream used by entry points that take host arrays; those entry points
// synchronise it before returning.  One per device, created on first use.
cudaStream_t host_api_stream();

// Owning device allocation (cudaMalloc / cudaFree).
template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
  cudaError_t upload(const T *h, size_t count, cudaStream_t s) {
    cudaError_t e = alloc(count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  cudaError_t upload(const std::vector<T> &v, cudaStream_t s) {
    return upload(v.data(), v.size(), s);
  }
  T *release() {
    T *q = p;
    p = nullptr;
    n = 0;
    return q;
  }
};

inline int cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return kOk;
  return set_error(e == cudaErrorMemoryAllocation ? kOutOfMemory : kCudaError,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

#define NAPMO_TRY_CUDA(expr, what)                                   \
  do {                                                               \
    cudaError_t _e = (expr);                                         \
    if (_e != cudaSuccess) return ::napmo::cuda_status(_e, (what));  \
  } while (0)

// Runs `f` (returning int status); converts C++ exceptions to kInvalidArgument.
template <class F>
int guarded(F &&f) {
  clear_error();
  try {
    return f();
  } catch (const std::exception &ex) {
    return set_error(kInvalidArgument, ex.what());
  } catch (...) {
    return set_error(kInvalidArgument, "unknown C++ exception");
  }
}

}  // namespace napmo
