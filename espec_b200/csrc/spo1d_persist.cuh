// spo1d_persist.cuh -- the whole uneven-size batch in ONE persistent launch.
//
// A CTA of kPersistThreads threads claims work items from a device counter
// until none is left.  An item is a group of packets of one size class that
// fills the CTA: 256 / T packets of T = N/P threads each (eight 256- or
// 384-point packets, four 512/768, two 1024/1536, one 2048), each group
// with its own slice of shared memory and its own hardware barrier.  Items
// are ordered by decreasing cost on the host (longest processing time
// first), so the last items to start are the short ones and no size class
// leaves a tail of idle SMs.  A claim is one atomicAdd: nothing waits on
// another CTA, so the claim loop needs no time-out and ends when the counter
// passes the item count.
#pragma once
#include "spo1d_launch.cuh"

namespace espec {

constexpr int kPersistThreads = 256;

struct SpoItem {
  int cls;    // size class (index into the plan set of the kernel)
  int first;  // first packet of the item in the packet list
  int count;  // packets of the item (<= kPersistThreads / T of its class)
};

template <typename R>
struct SpoPersistArgs {
  SpoArgs<R> a;            // tables, psi0/psi_out, C(t); a.pk = packets in item order
  const SpoItem* items;    // decreasing cost
  int nitems;
  unsigned int* next;      // claim counter, zero before the launch
};

constexpr size_t round16(size_t b) { return (b + 15) / 16 * 16; }

// the plan and table location of each size class in the persistent kernel:
// the per-size default variants of the per-class kernels (spo1d.cu)
template <typename R, int N>
struct PersistVariant {
  static constexpr int v = sizeof(R) == 8
                               ? ((N == 1024 || N == 1536 || N == 2048) ? 0 : 2)
                               : (N == 512 || N == 1536 ? 3 : (N == 1024 ? 1 : (N == 2048 ? 0 : 2)));
  using PL = typename VariantPlan<N, v>::type;
  static constexpr int kTab = VariantTab<v>::value;
  static constexpr int G = kPersistThreads / PL::T;  // packets per item
  static constexpr size_t group_smem = round16(spo1d_smem_bytes<R, PL, kTab>());
  static constexpr size_t smem = group_smem * G;
  static_assert(kPersistThreads % PL::T == 0, "a group must divide the CTA");
};

// size classes of the persistent kernel, in class-index order (4096-point
// packets, with 16 points per thread, run in the per-class kernels only:
// their register demand would spill in every class of the shared kernel)
constexpr int kPersistClasses = 7;
constexpr int kPersistSizes[kPersistClasses] = {256, 384, 512, 768, 1024, 1536, 2048};

template <typename R>
constexpr size_t persist_smem_bytes() {
  size_t m = PersistVariant<R, 256>::smem;
  m = m > PersistVariant<R, 384>::smem ? m : PersistVariant<R, 384>::smem;
  m = m > PersistVariant<R, 512>::smem ? m : PersistVariant<R, 512>::smem;
  m = m > PersistVariant<R, 768>::smem ? m : PersistVariant<R, 768>::smem;
  m = m > PersistVariant<R, 1024>::smem ? m : PersistVariant<R, 1024>::smem;
  m = m > PersistVariant<R, 1536>::smem ? m : PersistVariant<R, 1536>::smem;
  m = m > PersistVariant<R, 2048>::smem ? m : PersistVariant<R, 2048>::smem;
  return m;
}

// Not inlined: each class's time loop is register-allocated as its own
// function, as in its per-class kernel; the call costs once per item.
template <typename R, int N>
__device__ __noinline__ void persist_item(const SpoArgs<R>& a, const SpoItem it,
                                          unsigned char* smem) {
  using V = PersistVariant<R, N>;
  constexpr int T = V::PL::T;
  const int g = threadIdx.x / T;
  if (g < it.count) {
    // barrier 0 when the group is the whole CTA, else g + 1 (T = 64, 128);
    // groups of one warp synchronise with __syncwarp
    const int bar = V::G == 1 ? 0 : g + 1;
    spo_packet<R, typename V::PL, false, V::kTab>(a, a.pk[it.first + g], threadIdx.x - g * T,
                                                  smem + g * V::group_smem, bar);
  }
}

template <typename R>
__global__ void __launch_bounds__(kPersistThreads, 1) spo1d_persistent(SpoPersistArgs<R> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  for (;;) {
    __syncthreads();  // every group left the previous item before s_item changes
    if (threadIdx.x == 0) s_item = (int)atomicAdd(p.next, 1u);
    __syncthreads();
    const int i = s_item;
    if (i >= p.nitems) return;
    const SpoItem it = p.items[i];
    switch (it.cls) {
      case 0: persist_item<R, 256>(p.a, it, smem_raw); break;
      case 1: persist_item<R, 384>(p.a, it, smem_raw); break;
      case 2: persist_item<R, 512>(p.a, it, smem_raw); break;
      case 3: persist_item<R, 768>(p.a, it, smem_raw); break;
      case 4: persist_item<R, 1024>(p.a, it, smem_raw); break;
      case 5: persist_item<R, 1536>(p.a, it, smem_raw); break;
      default: persist_item<R, 2048>(p.a, it, smem_raw); break;
    }
  }
}

// host side (spo1d_persist.cu)
int persist_class(int n);            // class index of size n, -1 if none
int persist_group(int n, bool fp64); // packets per item of size n
// variant of size n inside the persistent kernel (its final-layout table)
int persist_variant(int n, bool fp64);
cudaError_t spo_persist_launch_f64(const SpoPersistArgs<double>& p, cudaStream_t st);
cudaError_t spo_persist_launch_f32(const SpoPersistArgs<float>& p, cudaStream_t st);

}  // namespace espec
