// spo1d_persist.cu -- instantiations and host launch of the persistent
// uneven-size split-operator kernel (spo1d_persist.cuh).
#include "spo1d_persist.cuh"

namespace espec {

static_assert(persist_smem_bytes<double>() <= kMaxSmem, "FP64 persistent kernel exceeds shared memory");
static_assert(persist_smem_bytes<float>() <= kMaxSmem, "FP32 persistent kernel exceeds shared memory");

int persist_class(int n) {
  for (int i = 0; i < kPersistClasses; ++i)
    if (kPersistSizes[i] == n) return i;
  return -1;
}

template <typename R>
static void class_info(int n, int& g, int& v) {
  switch (n) {
    case 256: g = PersistVariant<R, 256>::G; v = PersistVariant<R, 256>::v; break;
    case 384: g = PersistVariant<R, 384>::G; v = PersistVariant<R, 384>::v; break;
    case 512: g = PersistVariant<R, 512>::G; v = PersistVariant<R, 512>::v; break;
    case 768: g = PersistVariant<R, 768>::G; v = PersistVariant<R, 768>::v; break;
    case 1024: g = PersistVariant<R, 1024>::G; v = PersistVariant<R, 1024>::v; break;
    case 1536: g = PersistVariant<R, 1536>::G; v = PersistVariant<R, 1536>::v; break;
    case 2048: g = PersistVariant<R, 2048>::G; v = PersistVariant<R, 2048>::v; break;
    default: g = 0; v = 0; break;
  }
}

int persist_group(int n, bool fp64) {
  int g = 0, v = 0;
  if (fp64) class_info<double>(n, g, v);
  else class_info<float>(n, g, v);
  return g;
}

int persist_variant(int n, bool fp64) {
  int g = 0, v = 0;
  if (fp64) class_info<double>(n, g, v);
  else class_info<float>(n, g, v);
  return v;
}

// one CTA per SM slot the occupancy calculator allows (one, with the
// register budget of the FP64 plans), never more CTAs than items
template <typename R>
static cudaError_t persist_launch(const SpoPersistArgs<R>& p, cudaStream_t st) {
  constexpr size_t smem = persist_smem_bytes<R>();
  static DeviceFlags attr;
  cudaError_t e = set_max_smem_once(attr, spo1d_persistent<R>, smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spo1d_persistent<R>,
                                                         kPersistThreads, smem)) != cudaSuccess)
    return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const long slots = (long)sms * per_sm;
  const int grid = (int)(p.nitems < slots ? p.nitems : slots);
  if (grid < 1) return cudaSuccess;
  spo1d_persistent<R><<<grid, kPersistThreads, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t spo_persist_launch_f64(const SpoPersistArgs<double>& p, cudaStream_t st) {
  return persist_launch<double>(p, st);
}
cudaError_t spo_persist_launch_f32(const SpoPersistArgs<float>& p, cudaStream_t st) {
  return persist_launch<float>(p, st);
}

}  // namespace espec
