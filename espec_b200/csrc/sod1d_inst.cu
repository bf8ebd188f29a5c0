// kernel instantiations of the FP64 second-order-differences propagator
#include "sod1d.cuh"
#include "spo1d_launch.cuh"

namespace espec {

template <class PL, int kAbs>
static cudaError_t launch_sod_one(const SodArgs& a, int nblocks, cudaStream_t st) {
  constexpr size_t smem = sod1d_smem_bytes<PL>();
  if constexpr (smem > kMaxSmem) {
    return cudaErrorInvalidConfiguration;  // size rejected at plan creation
  } else {
    auto kern = sod1d_kernel<PL, kAbs>;
    static DeviceFlags attr_set;
    cudaError_t e = set_max_smem_once(attr_set, kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<nblocks, PL::T, smem, st>>>(a);
    return cudaGetLastError();
  }
}

template <int N>
static cudaError_t launch_sod_n(int kabs, const SodArgs& a, int nblocks, cudaStream_t st) {
  using PL = typename DefaultPlan<N>::type;
  switch (kabs) {
    case 1: return launch_sod_one<PL, 1>(a, nblocks, st);
    case 2: return launch_sod_one<PL, 2>(a, nblocks, st);
    default: return launch_sod_one<PL, 0>(a, nblocks, st);
  }
}

cudaError_t sod_launch(int n, int kabs, const SodArgs& a, int nblocks, cudaStream_t st) {
  switch (n) {
    case 256: return launch_sod_n<256>(kabs, a, nblocks, st);
    case 384: return launch_sod_n<384>(kabs, a, nblocks, st);
    case 512: return launch_sod_n<512>(kabs, a, nblocks, st);
    case 768: return launch_sod_n<768>(kabs, a, nblocks, st);
    case 1024: return launch_sod_n<1024>(kabs, a, nblocks, st);
    case 1536: return launch_sod_n<1536>(kabs, a, nblocks, st);
    case 2048: return launch_sod_n<2048>(kabs, a, nblocks, st);
    default: return cudaErrorInvalidValue;
  }
}

bool sod_size_supported(int n) {
  switch (n) {
    case 256: return sod1d_smem_bytes<DefaultPlan<256>::type>() <= kMaxSmem;
    case 384: return sod1d_smem_bytes<DefaultPlan<384>::type>() <= kMaxSmem;
    case 512: return sod1d_smem_bytes<DefaultPlan<512>::type>() <= kMaxSmem;
    case 768: return sod1d_smem_bytes<DefaultPlan<768>::type>() <= kMaxSmem;
    case 1024: return sod1d_smem_bytes<DefaultPlan<1024>::type>() <= kMaxSmem;
    case 1536: return sod1d_smem_bytes<DefaultPlan<1536>::type>() <= kMaxSmem;
    case 2048: return sod1d_smem_bytes<DefaultPlan<2048>::type>() <= kMaxSmem;
    default: return false;
  }
}

}  // namespace espec
