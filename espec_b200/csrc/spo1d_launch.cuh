// spo1d_launch.cuh -- launch helpers and the variant registry of the batched
// 1D split-operator kernel.  A variant fixes the radix plan, where the
// per-point tables live and the register budget (minimum resident CTAs per
// SM); the autotuner measures them and picks one per packet size.
#pragma once
#include "spo1d.cuh"

namespace espec {

// alternative plans (4 points per thread, radix-4 stages) for powers of two
template <int N>
struct AltPlan {
  using type = typename DefaultPlan<N>::type;
};
template <> struct AltPlan<256>  { using type = Plan<256, 4, 4, 4, 4, 4>; };
template <> struct AltPlan<512>  { using type = Plan<512, 4, 4, 4, 4, 4, 2>; };
template <> struct AltPlan<1024> { using type = Plan<1024, 4, 4, 4, 4, 4, 4>; };
template <> struct AltPlan<2048> { using type = Plan<2048, 4, 4, 4, 4, 4, 4, 2>; };
template <> struct AltPlan<4096> { using type = Plan<4096, 8, 8, 8, 8, 8>; };

constexpr int kNumVariants = 4;

template <typename R, class PL, bool kQuirk, int kTab, int kMinB>
static cudaError_t launch_one(const SpoArgs<R>& a, int nblocks, cudaStream_t st) {
  auto kern = spo1d_kernel<R, PL, false, kQuirk, kTab, kMinB>;
  const size_t smem = spo1d_smem_bytes<R, PL, kTab>();
  static bool attr_set = false;  // one flag per instantiation
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  kern<<<nblocks, PL::T, smem, st>>>(a);
  return cudaGetLastError();
}

// minimum resident CTAs that caps registers per thread at RegCap
template <class PL, int RegCap>
struct MinBlocks {
  static constexpr int v = (65536 / (RegCap * PL::T)) < 1 ? 1 : (65536 / (RegCap * PL::T));
};

// variant v of size N:
//   0: default plan, tables in registers, <= 255 registers
//   1: default plan, tables in shared memory, <= 168 registers
//   2: default plan, tables in shared memory, <= 128 registers
//   3: alternative plan (radix-4, 4 points/thread for powers of two), tables
//      in registers, <= 128 registers
template <typename R, int N>
static cudaError_t launch_variant(int v, const SpoArgs<R>& a, int nblocks, bool quirk,
                                  cudaStream_t st) {
  using D = typename DefaultPlan<N>::type;
  using A = typename AltPlan<N>::type;
  if constexpr (sizeof(R) == 8) {
    if (quirk) return launch_one<R, D, true, 0, 1>(a, nblocks, st);
  }
  switch (v) {
    case 1: return launch_one<R, D, false, 1, MinBlocks<D, 168>::v>(a, nblocks, st);
    case 2: return launch_one<R, D, false, 1, MinBlocks<D, 128>::v>(a, nblocks, st);
    case 3: return launch_one<R, A, false, 0, MinBlocks<A, 128>::v>(a, nblocks, st);
    default: return launch_one<R, D, false, 0, 1>(a, nblocks, st);
  }
}

// per translation unit entry points (spo1d_inst_*.cu)
cudaError_t spo_launch_f32_pow2(int n, int v, const SpoArgs<float>& a, int nblocks, cudaStream_t st);
cudaError_t spo_launch_f32_r3(int n, int v, const SpoArgs<float>& a, int nblocks, cudaStream_t st);
cudaError_t spo_launch_f64_pow2(int n, int v, const SpoArgs<double>& a, int nblocks, bool quirk,
                                cudaStream_t st);
cudaError_t spo_launch_f64_r3(int n, int v, const SpoArgs<double>& a, int nblocks, bool quirk,
                              cudaStream_t st);

}  // namespace espec
