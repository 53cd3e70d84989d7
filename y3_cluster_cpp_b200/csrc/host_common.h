// host_common.h -- host-side helpers shared by the y3b C-ABI implementation:
// thread-local error messages, status propagation without exceptions across
// the C boundary, launch accounting and a small RAII device buffer.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <new>
#include <string>
#include <vector>

#include "../../include/y3b.h"

namespace y3b {

void set_error(const char* fmt, ...);
void clear_error();
extern std::atomic<unsigned long long> g_launches;

inline void
count_launch(unsigned n = 1)
{
  g_launches.fetch_add(n, std::memory_order_relaxed);
}

// Returns Y3B_ERR_CUDA with a message if e is a CUDA error.
inline int
cuda_status(cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return Y3B_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? Y3B_ERR_NOMEM : Y3B_ERR_CUDA;
}

#define Y3B_TRY(expr)                     \
  do {                                    \
    int _rc = (expr);                     \
    if (_rc != Y3B_OK) return _rc;        \
  } while (0)

#define Y3B_CUDA(expr) Y3B_TRY(::y3b::cuda_status((expr), #expr))

// Checks that a usable sm_100 device is current.
int require_device();

// Minimal owning device buffer (no exceptions; check ok()).
template <typename T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  int alloc(size_t n)
  {
    if (n <= cap_) {
      n_ = n;
      return Y3B_OK;
    }
    reset();
    if (n == 0) return Y3B_OK;
    Y3B_CUDA(cudaMalloc(&p_, n * sizeof(T)));
    cap_ = n_ = n;
    return Y3B_OK;
  }
  int upload(const T* h, size_t n, cudaStream_t s = 0)
  {
    Y3B_TRY(alloc(n));
    if (n) Y3B_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return Y3B_OK;
  }
  void reset()
  {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = cap_ = 0;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0, cap_ = 0;
};

// Device status word for kernel-side checks (domain errors, timeouts).
int read_device_status(int* d_status, cudaStream_t s);
// Maps a device-side error code (DevErr) to a y3b_status and leaves its
// message for y3b_last_error().
int device_status_rc(int code);

}  // namespace y3b
