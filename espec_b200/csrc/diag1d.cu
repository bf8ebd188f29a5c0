// diag1d.cu -- per-packet energy and norm of the current wave functions of a
// plan, FP64, on the GPU (EFFT4 of eigenergfft.f:58-100 and the norm
// FCORREL(U,U)+FCORREL(V,V) of pspofft.f:96-98):
//   E = sum V (u^2 + v^2) + (1/N) sum_k TC(k) |F psi|_k^2,   norm = sum (u^2 + v^2)
// used for the printed partial C(t) rows and the drift check of the drop-ins.
#include <cuda_runtime.h>

#include "diag1d.cuh"
#include "espec_internal.h"
#include "spo1d_launch.cuh"

namespace espec {


template <class PL>
__global__ void __launch_bounds__(PL::T) diag1d_kernel(DiagArgs a) {
  using R = double;
  constexpr int N = PL::N, P = PL::P, T = PL::T, NW = (T + 31) / 32;
  using Th = SpoThread<R, PL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<R>* bufs = reinterpret_cast<cpx<R>*>(smem_raw);
  double* red = reinterpret_cast<double*>(bufs + Th::NBUF * N);  // [3][NW]
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const SpoPacket pk = a.pk[blockIdx.x];
  const int base = pk.off;
  Th th;
  th.init_twiddles(t);
  cpx<R> v[P];
  double epot = 0.0, nrm = 0.0, ekin = 0.0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int x = base + Th::x_pos(t, j);
    const double2 p = a.psi[x];
    v[j] = mk(p.x, p.y);
    const double vp = a.vpot[x];
    epot += p.x * vp * p.x + p.y * vp * p.y;
    nrm += p.x * p.x + p.y * p.y;
  }
  th.template forward<0>(v, bufs, t);
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int f = a.kfreq[Th::final_pos(t, j)];
    ekin += a.tc[base + f] * (v[j].x * v[j].x + v[j].y * v[j].y);
  }
  ekin /= (double)N;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    epot += __shfl_xor_sync(0xffffffffu, epot, o);
    nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    ekin += __shfl_xor_sync(0xffffffffu, ekin, o);
  }
  __syncthreads();  // exchange buffers may still be read by other warps
  if (lane == 0) {
    red[warp] = epot;
    red[NW + warp] = nrm;
    red[2 * NW + warp] = ekin;
  }
  __syncthreads();
  if (t == 0) {
    double e1 = 0, e2 = 0, n1 = 0;
    for (int i = 0; i < NW; ++i) {
      e1 += red[i];
      n1 += red[NW + i];
      e2 += red[2 * NW + i];
    }
    a.out[pk.c_off] = make_double2(e1 + e2, n1);
  }
}

template <int N>
static cudaError_t launch_diag_n(const DiagArgs& a, int nblocks, cudaStream_t st) {
  using PL = typename DefaultPlan<N>::type;
  using Th = SpoThread<double, PL>;
  constexpr size_t smem = Th::NBUF * sizeof(cpx<double>) * N + 3 * sizeof(double) * ((PL::T + 31) / 32);
  if constexpr (smem > kMaxSmem) {
    return cudaErrorInvalidConfiguration;
  } else {
    auto kern = diag1d_kernel<PL>;
    static DeviceFlags attr_set;
    cudaError_t e = set_max_smem_once(attr_set, kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<nblocks, PL::T, smem, st>>>(a);
    return cudaGetLastError();
  }
}

// the diagnostic FFT always uses DefaultPlan<N>, whatever variant the
// propagation kernel of the same size class runs; kfreq is built for it
cudaError_t diag_launch(int n, const DiagArgs& a, int nblocks, cudaStream_t st) {
  switch (n) {
    case 256: return launch_diag_n<256>(a, nblocks, st);
    case 384: return launch_diag_n<384>(a, nblocks, st);
    case 512: return launch_diag_n<512>(a, nblocks, st);
    case 768: return launch_diag_n<768>(a, nblocks, st);
    case 1024: return launch_diag_n<1024>(a, nblocks, st);
    case 1536: return launch_diag_n<1536>(a, nblocks, st);
    case 2048: return launch_diag_n<2048>(a, nblocks, st);
    case 4096: return launch_diag_n<4096>(a, nblocks, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace espec
