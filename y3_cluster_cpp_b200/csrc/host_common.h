// host_common.h -- host-side helpers shared by the y3b C-ABI implementation:
// thread-local error messages, status propagation without exceptions across
// the C boundary, launch accounting and a small RAII device buffer.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
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

// Gauss-Legendre nodes and weights on [a, b] in FP64: Newton on P_n from the
// Tricomi start cos(pi (i + 3/4) / (n + 1/2)) to |dz| <= 1e-14, nodes in
// ascending order (p_operator_cuhre_t.hh:66-95, the grids of P_operator and
// ShearPrjFrozenPhysics).
inline void
gl_nodes_host(double a, double b, int n, std::vector<double>& x, std::vector<double>& w)
{
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = 3.14159265358979323846;
  const double mid = 0.5 * (a + b), hl = 0.5 * (b - a);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5)), z1, pp;
    int guard = 0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 0; j < n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j + 1.0) * z * p2 - j * p3) / (j + 1.0);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) > 1e-14 && ++guard < 100);
    x[i] = mid - hl * z;
    x[n - 1 - i] = mid + hl * z;
    w[i] = w[n - 1 - i] = 2.0 * hl / ((1.0 - z * z) * pp * pp);
  }
}

// Device status word for kernel-side checks (domain errors, timeouts).
int read_device_status(int* d_status, cudaStream_t s);
// Maps a device-side error code (DevErr) to a y3b_status and leaves its
// message for y3b_last_error().
int device_status_rc(int code);

}  // namespace y3b
