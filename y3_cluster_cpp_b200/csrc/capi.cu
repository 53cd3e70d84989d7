// capi.cu -- C-ABI plumbing: thread-local error messages, device selection,
// launch accounting, device status words and the bounded-wait self-test.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "common.cuh"
#include "host_common.h"

namespace y3b {

std::atomic<unsigned long long> g_launches{0};

static thread_local std::string t_error;

void
set_error(const char* fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_error = buf;
}

void
clear_error()
{
  t_error.clear();
}

int
require_device()
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("no usable CUDA device: %s", cudaGetErrorString(e));
    return Y3B_ERR_CUDA;
  }
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a only", dev, major, minor);
    return Y3B_ERR_CUDA;
  }
  return Y3B_OK;
}

int
read_device_status(int* d_status, cudaStream_t s)
{
  int h = 0;
  Y3B_CUDA(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  Y3B_CUDA(cudaStreamSynchronize(s));
  return device_status_rc(h);
}

int
device_status_rc(int code)
{
  switch (code) {
    case kDevOk: return Y3B_OK;
    case kDevDomain:
      set_error("argument out of range in Interp1D (a z node lies outside distances/z or "
                "another unclamped table)");
      return Y3B_ERR_DOMAIN;
    case kDevTimeout:
      set_error("a bounded device-side wait ran out");
      return Y3B_ERR_TIMEOUT;
    case kDevNonFinite:
      set_error("a table entry is not finite (NaN or Inf)");
      return Y3B_ERR_DOMAIN;
    case kDevRange:
      set_error("mixed form: a point's Gaussian factors would leave the FP32 exponent range "
                "(sigma_int too small for the factorisation); evaluate it in FP64");
      return Y3B_ERR_RANGE;
    default:
      set_error("device-side shape check failed (code %d)", code);
      return Y3B_ERR_INVALID;
  }
}

// Waits on an mbarrier that nobody arrives at until `ns` nanoseconds of
// %globaltimer have passed, then records a timeout and returns.
__global__ void
wait_timeout_kernel(unsigned long long ns, int* status)
{
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t addr = static_cast<uint32_t>(__cvta_generic_to_shared(&bar));
  if (threadIdx.x == 0)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(addr) : "memory");
  __syncthreads();
  unsigned long long t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  uint32_t ok = 0;
  for (;;) {
    asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr)
      : "memory");
    if (ok) break;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > ns) break;
  }
  if (!ok && threadIdx.x == 0) set_err(status, kDevTimeout);
}

}  // namespace y3b

using namespace y3b;

extern "C" const char*
y3b_last_error(void)
{
  return t_error.c_str();
}

extern "C" int
y3b_version(void)
{
  return Y3B_VERSION;
}

extern "C" unsigned long long
y3b_launch_count(void)
{
  return g_launches.load();
}

extern "C" int
y3b_device_init(int device)
{
  clear_error();
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("no CUDA device available: %s", cudaGetErrorString(e));
    return Y3B_ERR_CUDA;
  }
  if (device < 0 || device >= n) {
    set_error("device %d outside [0, %d)", device, n);
    return Y3B_ERR_INVALID;
  }
  Y3B_CUDA(cudaSetDevice(device));
  return require_device();
}

extern "C" int
y3b_selftest_wait_timeout(int usec)
{
  clear_error();
  if (usec < 1 || usec > 5000000) {
    set_error("y3b_selftest_wait_timeout: usec must be in [1, 5e6]");
    return Y3B_ERR_INVALID;
  }
  Y3B_TRY(require_device());
  DevBuf<int> st;
  Y3B_TRY(st.alloc(1));
  Y3B_CUDA(cudaMemset(st.get(), 0, sizeof(int)));
  wait_timeout_kernel<<<1, 32>>>((unsigned long long)usec * 1000ull, st.get());
  count_launch();
  Y3B_CUDA(cudaGetLastError());
  return read_device_status(st.get(), 0);
}
