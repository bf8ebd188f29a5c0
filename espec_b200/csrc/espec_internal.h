// espec_internal.h -- error plumbing shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

namespace espec {
int set_error(int code, const char* msg);
int set_cuda_error(const char* what, cudaError_t e);
inline int ck(cudaError_t e, const char* what) {
  return e == cudaSuccess ? 0 : set_cuda_error(what, e);
}
}  // namespace espec
