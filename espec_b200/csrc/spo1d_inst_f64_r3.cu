// kernel instantiations: double, packet sizes 3 * 2^k
#include "spo1d_launch.cuh"
namespace espec {
cudaError_t spo_launch_f64_r3(int n, int v, const SpoArgs<double>& a, int nb, bool quirk, cudaStream_t st) {
  switch (n) {
    case 384: return launch_variant<double, 384>(v, a, nb, quirk, st);
    case 768: return launch_variant<double, 768>(v, a, nb, quirk, st);
    case 1536: return launch_variant<double, 1536>(v, a, nb, quirk, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace espec
