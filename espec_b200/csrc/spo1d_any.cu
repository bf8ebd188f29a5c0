// spo1d_any.cu -- the 1D split-operator, SOD-with-FFT and energy kernels for
// packet sizes outside the register plans of spo1d.cuh: any even size, FP64.
//
// eSPec's FFT (fft3d.f, Singleton's mixed-radix transform) takes any N, so
// its .PFSPO / .PFSOD runs do too.  Here one CTA owns one packet and keeps it
// in shared memory; the transform is a mixed-radix Stockham FFT (radices 4
// and 2, then every odd prime factor), natural order in and out, in which
// each output of a radix-r stage is the direct sum of its r inputs times
// twiddles from a per-size table w[e] = e^{+2 pi i e / N}.  A stage costs N r
// complex multiply-adds, so a size with a large prime factor is slow but
// exact to FP64 rounding.  The step, the tables (x order, and the kinetic
// table in natural FFT order) and the C(t) samples are those of the register
// kernels: spo_packet (spo1d.cuh) and sod1d_kernel (sod1d.cuh).
#include <cuda_runtime.h>

#include <cmath>

#include "diag1d.cuh"
#include "espec_gpu.h"
#include "espec_internal.h"
#include "sod1d.cuh"
#include "spo1d_any.cuh"
#include "spo1d_launch.cuh"

namespace espec {

bool any_plan(int n, AnyPlan& pl) {
  if (n < 4 || n % 2 || n > kAnyMaxN) return false;
  pl.n = n;
  pl.ns = 0;
  int m = n;
  auto push = [&](int r) {
    if (pl.ns >= kAnyMaxStages) return false;
    pl.r[pl.ns++] = r;
    m /= r;
    return true;
  };
  while (m % 4 == 0)
    if (!push(4)) return false;
  while (m % 2 == 0)
    if (!push(2)) return false;
  for (int p = 3; m > 1; p += 2)
    while (m % p == 0)
      if (!push(p)) return false;
  return true;
}

size_t any_smem_bytes(int n, int method) {
  const int nbuf = method == ESPEC_SOD ? 4 : 2;
  return (size_t)nbuf * n * sizeof(cpx<double>) + 3 * sizeof(double2) * (kAnyThreads / 32);
}

namespace {

// out = src transformed (forward: e^{+2 pi i jk/N}, inverse: conjugate, no
// scaling); src and dst are the two N-point buffers, the result lands in one
// of them (returned).  Ends with a CTA barrier.
__device__ cpx<double>* any_fft(const AnyPlan& pl, const double2* __restrict__ tw,
                                cpx<double>* src, cpx<double>* dst, bool inv) {
  const int n = pl.n, T = blockDim.x, t = threadIdx.x;
  int ns = 1;  // size of the sub-transforms done so far
  for (int s = 0; s < pl.ns; ++s) {
    const int r = pl.r[s], m = n / r, span = ns * r, tws = n / span;
    for (int o = t; o < n; o += T) {
      // output o = (j / ns) span + k ns + j % ns of input group j, digit k
      const int blk = o / span, rem = o - blk * span;
      const int k = rem / ns, jm = rem - k * ns;
      const int j = blk * ns + jm;
      int e1 = jm * tws + k * m;
      if (e1 >= n) e1 -= n;
      double sr = 0.0, si = 0.0;
      int e = 0;
      for (int q = 0; q < r; ++q) {
        const cpx<double> x = src[j + q * m];
        const double2 w = __ldg(tw + e);
        const double wi = inv ? -w.y : w.y;
        sr = fma(x.x, w.x, fma(-x.y, wi, sr));
        si = fma(x.x, wi, fma(x.y, w.x, si));
        e += e1;
        if (e >= n) e -= n;
      }
      dst[o] = mk(sr, si);
    }
    __syncthreads();
    cpx<double>* tmp = src;
    src = dst;
    dst = tmp;
    ns = span;
  }
  return src;
}

// sum over the CTA of (x, y); valid on thread 0.  red: [NW] scratch.
__device__ double2 cta_sum2(double x, double y, double2* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) / 32;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_xor_sync(0xffffffffu, x, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  if (lane == 0) red[warp] = make_double2(x, y);
  __syncthreads();
  double sx = 0.0, sy = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) {
      sx += red[i].x;
      sy += red[i].y;
    }
  __syncthreads();
  return make_double2(sx, sy);
}

__global__ void __launch_bounds__(kAnyThreads) spo_any_kernel(SpoArgs<double> a, AnyPlan pl,
                                                              const double2* tw, int quirk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using TB = Tab<double>;
  const int n = pl.n, t = threadIdx.x, T = blockDim.x;
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smem_raw);
  cpx<double>* b1 = b0 + n;
  double2* red = reinterpret_cast<double2*>(b1 + n);
  const SpoPacket pk = a.pk[blockIdx.x];
  const int base = pk.off;
  double2* cout = a.c_out + pk.c_off;
  double c0 = 0.0;
  for (int x = t; x < n; x += T) {
    const double2 p0 = a.psi_start ? a.psi_start[base + x] : a.psi0[base + x];
    b0[x] = mk(p0.x, p0.y);
    c0 += p0.x * p0.x + p0.y * p0.y;
  }
  if (!a.psi_start) {
    const double2 c = cta_sum2(c0, 0.0, red);
    if (t == 0) cout[0] = make_double2(c.x, 0.0);
  }
  bool finite = true;
  cpx<double>* v = b0;
  for (int step = 1; step <= a.nsteps; ++step) {
    const TB::phase_t* ph = step == 1 ? a.tab.h : a.tab.g;
    for (int x = t; x < n; x += T) v[x] = TB::apply(ph[base + x], v[x]);
    __syncthreads();
    cpx<double>* f = any_fft(pl, tw, v, v == b0 ? b1 : b0, false);
    for (int x = t; x < n; x += T) {
      if (quirk) {  // spofft.f:148-154 as written: V(I) uses the updated U(I)
        const double c = a.kq_c[base + x], s = a.kq_s[base + x];
        const double un = c * f[x].x + s * f[x].y;
        const double vn = c * f[x].y - s * un;
        f[x] = mk(un * a.kq_scale, vn * a.kq_scale);
      } else {
        f[x] = TB::apply(a.tab.k[base + x], f[x]);
      }
    }
    __syncthreads();
    v = any_fft(pl, tw, f, f == b0 ? b1 : b0, true);
    double cr = 0.0, ci = 0.0;
    for (int x = t; x < n; x += T) {
      const cpx<double> w = a.tab.w[base + x];
      cr = fma(w.x, v[x].x, fma(-w.y, v[x].y, cr));
      ci = fma(w.x, v[x].y, fma(w.y, v[x].x, ci));
    }
    const double2 c = cta_sum2(cr, ci, red);
    if (t == 0) {
      finite = finite && isfinite(c.x) && isfinite(c.y);
      cout[step] = c;
    }
  }
  if (t == 0 && !finite && a.nonfinite) atomicAdd(a.nonfinite, 1);
  if (a.psi_out)
    for (int x = t; x < n; x += T) {
      const cpx<double> o = a.nsteps > 0 ? TB::apply(a.tab.hm[base + x], v[x]) : v[x];
      a.psi_out[base + x] = make_double2(o.x, o.y);
    }
}

// kabs: 0 none, 1 complex absorbing potential, 2 multiplicative mask
__global__ void __launch_bounds__(kAnyThreads) sod_any_kernel(SodArgs a, AnyPlan pl,
                                                              const double2* tw, int kabs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = pl.n, t = threadIdx.x, T = blockDim.x;
  cpx<double>* cur = reinterpret_cast<cpx<double>*>(smem_raw);
  cpx<double>* prev = cur + n;
  cpx<double>* f0 = prev + n;
  cpx<double>* f1 = f0 + n;
  double2* red = reinterpret_cast<double2*>(f1 + n);
  const SpoPacket pk = a.pk[blockIdx.x];
  const int base = pk.off;
  double2* cout = a.c_out + pk.c_off;
  double c0 = 0.0;
  for (int x = t; x < n; x += T) {
    const double2 p0 = a.psi_start ? a.psi_start[base + x] : a.psi0[base + x];
    cur[x] = mk(p0.x, p0.y);
    const double2 q = a.psi_start ? a.psi_prev_start[base + x] : p0;
    prev[x] = mk(q.x, q.y);
    c0 += p0.x * p0.x + p0.y * p0.y;
  }
  if (!a.psi_start) {
    const double2 c = cta_sum2(c0, 0.0, red);
    if (t == 0) cout[0] = make_double2(c.x, 0.0);
  }
  // dst <- dst - i f (V src + T src) [+ f ab src]; dst holds the older state
  auto sod_update = [&](const cpx<double>* src, cpx<double>* dst, double f) {
    for (int x = t; x < n; x += T) f0[x] = src[x];
    __syncthreads();
    cpx<double>* k = any_fft(pl, tw, f0, f1, false);
    for (int x = t; x < n; x += T) {
      const double kc = a.tab.kc[base + x];
      k[x] = mk(k[x].x * kc, k[x].y * kc);
    }
    __syncthreads();
    const cpx<double>* h = any_fft(pl, tw, k, k == f0 ? f1 : f0, true);
    for (int x = t; x < n; x += T) {
      const double vc = a.tab.vc[base + x];
      const double hx = fma(vc, src[x].x, h[x].x), hy = fma(vc, src[x].y, h[x].y);
      double ox = fma(f, hy, dst[x].x), oy = fma(-f, hx, dst[x].y);
      if (kabs == 1) {  // + f CST VABC src (sodfft.f:68-70)
        const double ab = f * a.tab.ab[base + x];
        ox = fma(ab, src[x].x, ox);
        oy = fma(ab, src[x].y, oy);
      } else if (kabs == 2) {
        const double msk = a.tab.ab[base + x];
        ox *= msk;
        oy *= msk;
      }
      dst[x] = mk(ox, oy);
    }
  };
  auto c_sample = [&](const cpx<double>* psi, int step) {
    double cr = 0.0, ci = 0.0;
    for (int x = t; x < n; x += T) {
      const cpx<double> w = a.tab.w[base + x];
      cr = fma(w.x, psi[x].x, fma(-w.y, psi[x].y, cr));
      ci = fma(w.x, psi[x].y, fma(w.y, psi[x].x, ci));
    }
    const double2 c = cta_sum2(cr, ci, red);
    if (t == 0) cout[step] = c;
  };
  bool cur_newest = true;
  int step = 2;
  if (a.psi_start) {
    step = 1;
  } else if (a.nsteps >= 1) {
    // start-up (psodfft.f:120-152): E = psi0 - i/2 H psi0 ; psi1 = psi0 - i/2 H E
    sod_update(cur, prev, 0.5);
    sod_update(prev, cur, 0.5);
    for (int x = t; x < n; x += T) {
      const double2 p0 = a.psi0[base + x];
      prev[x] = mk(p0.x, p0.y);
    }
    c_sample(cur, 1);
  }
  for (; step + 1 <= a.nsteps; step += 2) {
    sod_update(cur, prev, 1.0);
    c_sample(prev, step);
    sod_update(prev, cur, 1.0);
    c_sample(cur, step + 1);
  }
  if (step <= a.nsteps) {
    sod_update(cur, prev, 1.0);
    c_sample(prev, step);
    cur_newest = false;
  }
  if (a.psi_out) {
    const cpx<double>* nw = cur_newest ? cur : prev;
    const cpx<double>* od = cur_newest ? prev : cur;
    for (int x = t; x < n; x += T) {
      a.psi_out[base + x] = make_double2(nw[x].x, nw[x].y);
      if (a.psi_prev_out) a.psi_prev_out[base + x] = make_double2(od[x].x, od[x].y);
    }
  }
}

// (EFFT4 energy, norm) of the current state, as diag1d_kernel
__global__ void __launch_bounds__(kAnyThreads) diag_any_kernel(DiagArgs a, AnyPlan pl,
                                                               const double2* tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = pl.n, t = threadIdx.x, T = blockDim.x;
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smem_raw);
  cpx<double>* b1 = b0 + n;
  double2* red = reinterpret_cast<double2*>(b1 + n);
  const SpoPacket pk = a.pk[blockIdx.x];
  const int base = pk.off;
  double epot = 0.0, nrm = 0.0, ekin = 0.0;
  for (int x = t; x < n; x += T) {
    const double2 p = a.psi[base + x];
    b0[x] = mk(p.x, p.y);
    const double vp = a.vpot[base + x];
    epot += p.x * vp * p.x + p.y * vp * p.y;
    nrm += p.x * p.x + p.y * p.y;
  }
  __syncthreads();
  const cpx<double>* f = any_fft(pl, tw, b0, b1, false);
  for (int x = t; x < n; x += T) ekin += a.tc[base + x] * (f[x].x * f[x].x + f[x].y * f[x].y);
  ekin /= (double)n;
  const double2 s = cta_sum2(epot, nrm, red);
  const double2 k = cta_sum2(ekin, 0.0, red + kAnyThreads / 32);
  if (t == 0) a.out[pk.c_off] = make_double2(s.x + k.x, s.y);
}

template <class K, class... A>
cudaError_t any_launch(K kern, DeviceFlags& flags, int n, int method, int nblocks,
                       cudaStream_t st, const A&... args) {
  const size_t smem = any_smem_bytes(n, method);
  if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
  cudaError_t e = set_max_smem_once(flags, kern, kMaxSmem);
  if (e != cudaSuccess) return e;
  kern<<<nblocks, kAnyThreads, smem, st>>>(args...);
  return cudaGetLastError();
}

}  // namespace

cudaError_t spo_any_launch(const SpoArgs<double>& a, const AnyPlan& pl, const double2* tw,
                           bool quirk, int nblocks, cudaStream_t st) {
  static DeviceFlags f;
  return any_launch(spo_any_kernel, f, pl.n, ESPEC_SPO, nblocks, st, a, pl, tw, quirk ? 1 : 0);
}

cudaError_t sod_any_launch(const SodArgs& a, const AnyPlan& pl, const double2* tw, int kabs,
                           int nblocks, cudaStream_t st) {
  static DeviceFlags f;
  return any_launch(sod_any_kernel, f, pl.n, ESPEC_SOD, nblocks, st, a, pl, tw, kabs);
}

cudaError_t diag_any_launch(const DiagArgs& a, const AnyPlan& pl, const double2* tw, int nblocks,
                            cudaStream_t st) {
  static DeviceFlags f;
  return any_launch(diag_any_kernel, f, pl.n, ESPEC_SPO, nblocks, st, a, pl, tw);
}

// w[e] = (cos 2 pi e / N, sin 2 pi e / N), from long-double cosines and sines
void any_twiddles(int n, double2* w) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int e = 0; e < n; ++e) {
    const long double a = 2.0L * pi * (long double)e / (long double)n;
    w[e] = make_double2((double)cosl(a), (double)sinl(a));
  }
}

}  // namespace espec
