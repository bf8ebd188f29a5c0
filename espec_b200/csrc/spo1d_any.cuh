// spo1d_any.cuh -- 1D packets of any even size (spo1d_any.cu): the radix
// plan of the shared-memory Stockham FFT and the launches.
#pragma once
#include <cuda_runtime.h>

#include "diag1d.cuh"
#include "espec_gpu.h"
#include "sod1d.cuh"
#include "spo1d.cuh"

namespace espec {

constexpr int kAnyThreads = 256;
constexpr int kAnyMaxStages = 32;
constexpr int kAnyMaxN = 1 << 16;  // the shared-memory bound below is the tighter one

struct AnyPlan {
  int n, ns;               // size, number of stages
  int r[kAnyMaxStages];    // radix of each stage (product n)
};

// radices for size n (even, 4 <= n <= kAnyMaxN); false if n has none
bool any_plan(int n, AnyPlan& pl);
// dynamic shared memory of one CTA: ESPEC_SPO (and the energies) hold two
// N-point buffers, ESPEC_SOD four
size_t any_smem_bytes(int n, int method);
void any_twiddles(int n, double2* w);
cudaError_t spo_any_launch(const SpoArgs<double>& a, const AnyPlan& pl, const double2* tw,
                           bool quirk, int nblocks, cudaStream_t st);
cudaError_t sod_any_launch(const SodArgs& a, const AnyPlan& pl, const double2* tw, int kabs,
                           int nblocks, cudaStream_t st);
cudaError_t diag_any_launch(const DiagArgs& a, const AnyPlan& pl, const double2* tw, int nblocks,
                            cudaStream_t st);

}  // namespace espec
