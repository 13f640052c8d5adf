// capi.cu -- library-level entry points of the C ABI: version, thread-local
// error messages, device query and the FP64 throughput probe used as the
// measured roofline peak of the FP64 kernels.
#include <stdarg.h>
#include <stdio.h>

#include "psb_common.cuh"

namespace psb {

static thread_local char g_last_error[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int check_cuda(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(PSB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return PSB_OK;
}

// Eight independent FMA chains per thread; the sink write keeps them live.
__global__ void __launch_bounds__(256) fp64_fma_kernel(int iters, double* sink) {
  double a = 1.0 + 1e-9 * threadIdx.x, b = 0.999999999;
  double c[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i] = 0.5 * i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) c[i] = fma(c[i], b, a);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i];
  if (s == 1234.5678) sink[blockIdx.x] = s;
}

}  // namespace psb

using namespace psb;

extern "C" int psb_abi_version(void) { return PSB_ABI_VERSION; }

extern "C" const char* psb_last_error(void) { return g_last_error; }

extern "C" int psb_device_arch(int* arch) {
  if (!arch) return set_error(PSB_ERR_INVALID, "psb_device_arch: null pointer");
  int dev = 0, major = 0, minor = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (e != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "psb_device_arch: %s", cudaGetErrorString(e));
  *arch = major * 10 + minor;
  return PSB_OK;
}

extern "C" int psb_probe_fp64_fma(int blocks, int iters, double* d_sink, float* ms,
                                  void* stream) {
  if (blocks <= 0 || iters <= 0 || !d_sink || !ms)
    return set_error(PSB_ERR_INVALID, "psb_probe_fp64_fma: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return check_cuda("psb_probe_fp64_fma: event");
  cudaEventRecord(e0, st);
  fp64_fma_kernel<<<blocks, 256, 0, st>>>(iters, d_sink);
  cudaEventRecord(e1, st);
  cudaError_t err = cudaEventSynchronize(e1);
  float t = 0.f;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess)
    return set_error(PSB_ERR_CUDA, "psb_probe_fp64_fma: %s", cudaGetErrorString(err));
  *ms = t;
  return check_cuda("psb_probe_fp64_fma");
}
