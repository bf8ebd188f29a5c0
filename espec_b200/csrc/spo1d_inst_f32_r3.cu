// kernel instantiations: float, packet sizes 3 * 2^k
#include "spo1d_launch.cuh"
namespace espec {
cudaError_t spo_launch_f32_r3(int n, int v, const SpoArgs<float>& a, int nb, cudaStream_t st) {
  switch (n) {
    case 384: return launch_variant<float, 384>(v, a, nb, false, st);
    case 768: return launch_variant<float, 768>(v, a, nb, false, st);
    case 1536: return launch_variant<float, 1536>(v, a, nb, false, st);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace espec
