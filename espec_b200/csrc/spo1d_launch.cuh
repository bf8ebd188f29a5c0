// spo1d_launch.cuh -- launch helpers and the variant registry of the batched
// 1D split-operator kernel.  A variant fixes the radix plan, where the
// per-point tables live and the register budget (minimum resident CTAs per
// SM); the autotuner (espec_b200/autotune.py) measures them and the
// per-size defaults of spo1d.cu come from its results on B200.
#pragma once
#include "espec_internal.h"
#include "spo1d.cuh"

namespace espec {

// classic plans: largest radix first (the first exchanges are CTA-wide)
template <int N>
struct ClassicPlan;
template <> struct ClassicPlan<256>  { using type = Plan<256, 8, 8, 8, 4>; };
template <> struct ClassicPlan<512>  { using type = Plan<512, 8, 8, 8, 8>; };
template <> struct ClassicPlan<1024> { using type = Plan<1024, 8, 8, 8, 8, 2>; };
template <> struct ClassicPlan<2048> { using type = Plan<2048, 8, 8, 8, 8, 4>; };
template <> struct ClassicPlan<4096> { using type = Plan<4096, 16, 16, 16, 16>; };
template <> struct ClassicPlan<384>  { using type = Plan<384, 12, 12, 4, 4, 2>; };
template <> struct ClassicPlan<768>  { using type = Plan<768, 12, 12, 4, 4, 4>; };
template <> struct ClassicPlan<1536> { using type = Plan<1536, 12, 12, 4, 4, 4, 2>; };

// radix-4 plans (4 points per thread) for powers of two
template <int N>
struct AltPlan {
  using type = typename DefaultPlan<N>::type;
};
template <> struct AltPlan<256>  { using type = Plan<256, 4, 4, 4, 4, 4>; };
template <> struct AltPlan<512>  { using type = Plan<512, 4, 4, 4, 4, 4, 2>; };
template <> struct AltPlan<1024> { using type = Plan<1024, 4, 4, 4, 4, 4, 4>; };
template <> struct AltPlan<2048> { using type = Plan<2048, 4, 4, 4, 4, 4, 4, 2>; };
template <> struct AltPlan<4096> { using type = Plan<4096, 8, 8, 8, 8, 8>; };

constexpr int kNumVariants = 5;
constexpr size_t kMaxSmem = 227 * 1024;  // opt-in shared memory per CTA on sm_100

// minimum resident CTAs that caps registers per thread at RegCap
template <class PL, int RegCap>
struct MinBlocks {
  static constexpr int v = (65536 / (RegCap * PL::T)) < 1 ? 1 : (65536 / (RegCap * PL::T));
};

template <typename R, class PL, bool kQuirk, int kTab, int kMinB>
static cudaError_t launch_one(const SpoArgs<R>& a, int nblocks, cudaStream_t st) {
  constexpr size_t smem = spo1d_smem_bytes<R, PL, kTab>();
  if constexpr (smem > kMaxSmem) {
    return cudaErrorInvalidConfiguration;  // never selected: rejected by variant_fits
  } else {
    auto kern = spo1d_kernel<R, PL, false, kQuirk, kTab, kMinB>;
    static DeviceFlags attr_set;  // per instantiation, one bit per device
    cudaError_t e = set_max_smem_once(attr_set, kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<nblocks, PL::T, smem, st>>>(a);
    return cudaGetLastError();
  }
}

// variant v of size N:
//   0: warp-local plan, tables in registers
//   1: warp-local plan, tables in shared memory, <= 168 registers
//   2: classic plan, tables in registers
//   3: classic plan, tables in shared memory, <= 168 registers
//   4: radix-4 plan (4 points/thread for powers of two), tables in
//      registers, <= 128 registers
template <int N, int v>
struct VariantPlan {
  using type = typename DefaultPlan<N>::type;
};
template <int N> struct VariantPlan<N, 2> { using type = typename ClassicPlan<N>::type; };
template <int N> struct VariantPlan<N, 3> { using type = typename ClassicPlan<N>::type; };
template <int N> struct VariantPlan<N, 4> { using type = typename AltPlan<N>::type; };
template <int v> struct VariantTab {
  static constexpr int value = (v == 1 || v == 3) ? 1 : 0;
};
template <int v> struct VariantRegs {
  static constexpr int cap = v == 4 ? 128 : ((v == 1 || v == 3) ? 168 : 255);
};

template <typename R, int N, int v>
static cudaError_t launch_v(const SpoArgs<R>& a, int nblocks, cudaStream_t st) {
  using PL = typename VariantPlan<N, v>::type;
  return launch_one<R, PL, false, VariantTab<v>::value, MinBlocks<PL, VariantRegs<v>::cap>::v>(
      a, nblocks, st);
}

template <typename R, int N>
static cudaError_t launch_variant(int v, const SpoArgs<R>& a, int nblocks, bool quirk,
                                  cudaStream_t st) {
  if constexpr (sizeof(R) == 8) {
    if (quirk) return launch_one<R, typename DefaultPlan<N>::type, true, 0, 1>(a, nblocks, st);
  }
  switch (v) {
    case 1: return launch_v<R, N, 1>(a, nblocks, st);
    case 2: return launch_v<R, N, 2>(a, nblocks, st);
    case 3: return launch_v<R, N, 3>(a, nblocks, st);
    case 4: return launch_v<R, N, 4>(a, nblocks, st);
    default: return launch_v<R, N, 0>(a, nblocks, st);
  }
}

// shared memory of variant v of size N
template <typename R, int N, int v>
static size_t smem_v() {
  return spo1d_smem_bytes<R, typename VariantPlan<N, v>::type, VariantTab<v>::value>();
}
template <typename R, int N>
static size_t variant_smem(int v) {
  switch (v) {
    case 0: return smem_v<R, N, 0>();
    case 1: return smem_v<R, N, 1>();
    case 2: return smem_v<R, N, 2>();
    case 3: return smem_v<R, N, 3>();
    case 4: return smem_v<R, N, 4>();
    default: return 0;
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
