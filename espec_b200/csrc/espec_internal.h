// espec_internal.h -- error plumbing shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <string>

namespace espec {
int set_error(int code, const char* msg);
int set_cuda_error(const char* what, cudaError_t e);
// kinetic table of a 1D packet in FFT order (DIGT, dkeft.f:64-79)
void digt_1d(int n, double sh, double sm, double* tc);
// kinetic table of a 2D/3D grid in the reference's FFT order (dkeft.f:80-137
// as written with ESPEC_Q_DIGT_ND, else the outer sum of the axis tables)
void digt_nd_table(int ndim, const int* np, const double* sh, const double* sm, int quirks,
                   double* tc);
// the spectrum block SPECTRUMTD prints (spectrumtd.f:84-97) for FFTNT's
// output u + i v of 2^mf points
std::string spectrum_table(int mf, double dt, double de, const double* u, const double* v);
inline int ck(cudaError_t e, const char* what) {
  return e == cudaSuccess ? 0 : set_cuda_error(what, e);
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) applies to the current
// device only, so a kernel that needs more than 48 KB must have it set once
// on every device it runs on.  One bit per device ordinal below 64 records
// that; on higher ordinals the attribute is set before every launch.
struct DeviceFlags {
  std::atomic<unsigned long long> bits{0};
};
template <class K>
inline cudaError_t set_max_smem_once(DeviceFlags& f, K kern, size_t smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
  if (bit && (f.bits.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && bit) f.bits.fetch_or(bit, std::memory_order_release);
  return e;
}
}  // namespace espec
