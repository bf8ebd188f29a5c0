// cplx_io.cuh -- moving complex arrays between the interface form (separate
// real and imaginary float64 arrays: the reference's U/V and LNZVC columns)
// and the device form (interleaved double2).  Host transfers go through a
// contiguous (re | im) staging block owned by the plan, so each is one linear
// copy; device arguments are (de)interleaved in place by a kernel.
#pragma once
#include <cuda_runtime.h>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {

struct HostStage {
  double* d = nullptr;
  size_t bytes = 0;
  void release() {
    if (d) cudaFree(d);
    d = nullptr;
    bytes = 0;
  }
};

namespace {

__global__ void interleave_kernel(const double* re, const double* im, double2* out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_double2(re[i], im ? im[i] : 0.0);
}

__global__ void deinterleave_kernel(const double2* in, double* re, double* im, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    if (re) re[i] = v.x;
    if (im) im[i] = v.y;
  }
}

inline unsigned io_blocks(size_t n) {
  const size_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

#define IO_CK(call)                                          \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_); \
  } while (0)

inline int stage_reserve(HostStage& s, size_t bytes) {
  if (s.bytes >= bytes) return ESPEC_OK;
  s.release();
  IO_CK(cudaMalloc(&s.d, bytes));
  s.bytes = bytes;
  return ESPEC_OK;
}

// dst (device, n complex) <- (re, im) at `where`; im may be null (zero)
// a user pointer in host memory (synchronous or in-flight copies)
inline bool on_host(int where) { return where == ESPEC_MEM_HOST || where == ESPEC_MEM_HOST_ASYNC; }

inline int put_complex(HostStage& s, double2* dst, const double* re, const double* im, size_t n,
                       int where, cudaStream_t st) {
  if (n == 0) return ESPEC_OK;
  if (on_host(where)) {
    const int rc = stage_reserve(s, 16 * n);
    if (rc) return rc;
    IO_CK(cudaMemcpyAsync(s.d, re, 8 * n, cudaMemcpyHostToDevice, st));
    if (im) IO_CK(cudaMemcpyAsync(s.d + n, im, 8 * n, cudaMemcpyHostToDevice, st));
    re = s.d;
    im = im ? s.d + n : nullptr;
  }
  interleave_kernel<<<io_blocks(n), 256, 0, st>>>(re, im, dst, n);
  IO_CK(cudaGetLastError());
  return ESPEC_OK;
}

// (re, im) at `where` <- src (device, n complex); either output may be null
inline int get_complex(HostStage& s, const double2* src, double* re, double* im, size_t n,
                       int where, cudaStream_t st) {
  if ((!re && !im) || n == 0) return ESPEC_OK;
  if (!on_host(where)) {
    deinterleave_kernel<<<io_blocks(n), 256, 0, st>>>(src, re, im, n);
    IO_CK(cudaGetLastError());
    return ESPEC_OK;
  }
  const int rc = stage_reserve(s, 16 * n);
  if (rc) return rc;
  deinterleave_kernel<<<io_blocks(n), 256, 0, st>>>(src, s.d, s.d + n, n);
  IO_CK(cudaGetLastError());
  if (re) IO_CK(cudaMemcpyAsync(re, s.d, 8 * n, cudaMemcpyDeviceToHost, st));
  if (im) IO_CK(cudaMemcpyAsync(im, s.d + n, 8 * n, cudaMemcpyDeviceToHost, st));
  return ESPEC_OK;
}

#undef IO_CK

}  // namespace
}  // namespace espec
