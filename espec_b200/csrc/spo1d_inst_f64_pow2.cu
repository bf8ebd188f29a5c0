// kernel instantiations: double, power-of-two packet sizes
#include "spo1d_launch.cuh"
namespace espec {
cudaError_t spo_launch_f64_pow2(int n, int v, const SpoArgs<double>& a, int nb, bool quirk, cudaStream_t st) {
  switch (n) {
    case 256: return launch_variant<double, 256>(v, a, nb, quirk, st);
    case 512: return launch_variant<double, 512>(v, a, nb, quirk, st);
    case 1024: return launch_variant<double, 1024>(v, a, nb, quirk, st);
    case 2048: return launch_variant<double, 2048>(v, a, nb, quirk, st);
    case 4096: return launch_variant<double, 4096>(v, a, nb, quirk, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace espec
