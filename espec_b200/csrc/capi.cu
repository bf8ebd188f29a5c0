// capi.cu -- error state, version and device checks of libespecgpu.so.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {

static thread_local std::string g_last_error;

int set_error(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

int set_cuda_error(const char* what, cudaError_t e) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  g_last_error = buf;
  return e == cudaErrorMemoryAllocation ? ESPEC_ENOMEM : ESPEC_ECUDA;
}

}  // namespace espec

extern "C" const char* espec_last_error(void) { return espec::g_last_error.c_str(); }

extern "C" const char* espec_version(void) { return "espec_b200 0.1 (sm_100a)"; }

extern "C" int espec_device_ok(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return 0;
  return prop.major == 10 ? 1 : 0;
}
