// kernel instantiations: float, power-of-two packet sizes
#include "spo1d_launch.cuh"
namespace espec {
cudaError_t spo_launch_f32_pow2(int n, int v, const SpoArgs<float>& a, int nb, cudaStream_t st) {
  switch (n) {
    case 256: return launch_variant<float, 256>(v, a, nb, false, st);
    case 512: return launch_variant<float, 512>(v, a, nb, false, st);
    case 1024: return launch_variant<float, 1024>(v, a, nb, false, st);
    case 2048: return launch_variant<float, 2048>(v, a, nb, false, st);
    case 4096: return launch_variant<float, 4096>(v, a, nb, false, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace espec
