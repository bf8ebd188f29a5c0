// spo1d_any.cu -- the 1D split-operator, SOD-with-FFT and energy kernels for
// packet sizes outside the register plans of spo1d.cuh: any even size, FP64.
//
// eSPec's FFT (fft3d.f, Singleton's mixed-radix transform) takes any N, so
// its .PFSPO / .PFSOD runs do too.  Here one CTA owns one packet and keeps it
// in shared memory; the transform is a mixed-radix Stockham FFT (radices 4
// and 2, then every odd prime factor), natural order in and out: each thread
// takes one butterfly of a stage into registers, twiddles it from a per-size
// table w[e] = e^{+2 pi i e / N} and writes its r outputs (radix 2, 3, 4 and 5
// written out, other radices up to 16 as a direct sum in registers, larger
// primes output by output: N r complex multiply-adds for such a stage).  The step, the tables (x order, and the kinetic
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

// x * w, w given as (cos, sin) and conjugated for the inverse
__device__ __forceinline__ cpx<double> twid(cpx<double> x, double2 w, bool inv) {
  const double wi = inv ? -w.y : w.y;
  return mk(fma(x.x, w.x, -x.y * wi), fma(x.x, wi, x.y * w.x));
}
// i * x (forward) or -i * x (inverse)
__device__ __forceinline__ cpx<double> rot90(cpx<double> x, bool inv) {
  return inv ? mk(x.y, -x.x) : mk(-x.y, x.x);
}

// y_k = sum_q x_q w_R^{qk}, w_R = e^{+2 pi i/R} (conjugated for the
// inverse), in registers: the radix-2, 3, 4 and 5 butterflies written out,
// other radices up to kAnyRegRadix as the direct sum with the table's w_R
constexpr int kAnyRegRadix = 16;
template <int R>
__device__ __forceinline__ void dft_small(cpx<double>* x, const double2* __restrict__ tw, int n,
                                          bool inv) {
  if constexpr (R == 2) {
    const cpx<double> a = x[0], b = x[1];
    x[0] = mk(a.x + b.x, a.y + b.y);
    x[1] = mk(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    const cpx<double> a = mk(x[0].x + x[2].x, x[0].y + x[2].y);
    const cpx<double> b = mk(x[0].x - x[2].x, x[0].y - x[2].y);
    const cpx<double> c = mk(x[1].x + x[3].x, x[1].y + x[3].y);
    const cpx<double> d = rot90(mk(x[1].x - x[3].x, x[1].y - x[3].y), inv);
    x[0] = mk(a.x + c.x, a.y + c.y);
    x[2] = mk(a.x - c.x, a.y - c.y);
    x[1] = mk(b.x + d.x, b.y + d.y);
    x[3] = mk(b.x - d.x, b.y - d.y);
  } else if constexpr (R == 3) {
    const double2 w = __ldg(tw + n / 3);  // (cos 2pi/3, sin 2pi/3)
    const cpx<double> a = mk(x[1].x + x[2].x, x[1].y + x[2].y);
    const cpx<double> b = mk(x[1].x - x[2].x, x[1].y - x[2].y);
    const cpx<double> c = mk(fma(w.x, a.x, x[0].x), fma(w.x, a.y, x[0].y));
    const cpx<double> u = rot90(mk(w.y * b.x, w.y * b.y), inv);
    x[0] = mk(x[0].x + a.x, x[0].y + a.y);
    x[1] = mk(c.x + u.x, c.y + u.y);
    x[2] = mk(c.x - u.x, c.y - u.y);
  } else if constexpr (R == 5) {
    const double2 w1 = __ldg(tw + n / 5), w2 = __ldg(tw + 2 * (n / 5));
    const cpx<double> a1 = mk(x[1].x + x[4].x, x[1].y + x[4].y);
    const cpx<double> b1 = mk(x[1].x - x[4].x, x[1].y - x[4].y);
    const cpx<double> a2 = mk(x[2].x + x[3].x, x[2].y + x[3].y);
    const cpx<double> b2 = mk(x[2].x - x[3].x, x[2].y - x[3].y);
    const cpx<double> c1 = mk(x[0].x + w1.x * a1.x + w2.x * a2.x, x[0].y + w1.x * a1.y + w2.x * a2.y);
    const cpx<double> c2 = mk(x[0].x + w2.x * a1.x + w1.x * a2.x, x[0].y + w2.x * a1.y + w1.x * a2.y);
    const cpx<double> s1 = rot90(mk(w1.y * b1.x + w2.y * b2.x, w1.y * b1.y + w2.y * b2.y), inv);
    const cpx<double> s2 = rot90(mk(w2.y * b1.x - w1.y * b2.x, w2.y * b1.y - w1.y * b2.y), inv);
    x[0] = mk(x[0].x + a1.x + a2.x, x[0].y + a1.y + a2.y);
    x[1] = mk(c1.x + s1.x, c1.y + s1.y);
    x[4] = mk(c1.x - s1.x, c1.y - s1.y);
    x[2] = mk(c2.x + s2.x, c2.y + s2.y);
    x[3] = mk(c2.x - s2.x, c2.y - s2.y);
  }
}

// one Stockham stage of radix R (compile time) or r (run time): butterfly j
// takes x_q = src[j + q m], q < r, twiddles them by w_N^{(j % ns) q N/span},
// and writes its r-point DFT to dst[(j / ns) span + k ns + j % ns]
template <int R>
__device__ __forceinline__ void any_stage(const double2* __restrict__ tw, const cpx<double>* src,
                                          cpx<double>* dst, int n, int r, int ns, bool inv) {
  const int T = blockDim.x, t = threadIdx.x;
  const int m = n / r, span = ns * r, tws = n / span;
  for (int j = t; j < m; j += T) {
    const int jm = j % ns, base = (j / ns) * span + jm;
    if (R > 0 || r <= kAnyRegRadix) {
      constexpr int RR = R > 0 ? R : kAnyRegRadix;
      cpx<double> x[RR];
      const int e1 = jm * tws;  // < n / r
      int e = 0;
#pragma unroll
      for (int q = 0; q < RR; ++q) {
        if (R == 0 && q >= r) break;
        x[q] = src[j + q * m];
        if (q > 0) x[q] = twid(x[q], __ldg(tw + e), inv);
        e += e1;  // q e1 < n: no wrap
      }
      if constexpr (R > 0) {
        dft_small<R>(x, tw, n, inv);
#pragma unroll
        for (int k = 0; k < R; ++k) dst[base + k * ns] = x[k];
      } else {
        for (int k = 0; k < r; ++k) {  // direct sum with w_r^{qk} = w_N^{qk m}
          double sr = 0.0, si = 0.0;
          int f = 0;
          for (int q = 0; q < r; ++q) {
            const cpx<double> y = twid(x[q], __ldg(tw + f), inv);
            sr += y.x;
            si += y.y;
            f += k * m;
            if (f >= n) f -= n;
          }
          dst[base + k * ns] = mk(sr, si);
        }
      }
    } else {
      // a prime radix above kAnyRegRadix: each output from the r inputs
      for (int k = 0; k < r; ++k) {
        int e1 = jm * tws + k * m;
        if (e1 >= n) e1 -= n;
        double sr = 0.0, si = 0.0;
        int e = 0;
        for (int q = 0; q < r; ++q) {
          const cpx<double> y = twid(src[j + q * m], __ldg(tw + e), inv);
          sr += y.x;
          si += y.y;
          e += e1;
          if (e >= n) e -= n;
        }
        dst[base + k * ns] = mk(sr, si);
      }
    }
  }
}

// out = src transformed (forward: e^{+2 pi i jk/N}, inverse: conjugate, no
// scaling); src and dst are the two N-point buffers, the result lands in one
// of them (returned).  Ends with a CTA barrier.
__device__ cpx<double>* any_fft(const AnyPlan& pl, const double2* __restrict__ tw,
                                cpx<double>* src, cpx<double>* dst, bool inv) {
  const int n = pl.n;
  int ns = 1;  // size of the sub-transforms done so far
  for (int s = 0; s < pl.ns; ++s) {
    const int r = pl.r[s];
    switch (r) {
      case 2: any_stage<2>(tw, src, dst, n, r, ns, inv); break;
      case 3: any_stage<3>(tw, src, dst, n, r, ns, inv); break;
      case 4: any_stage<4>(tw, src, dst, n, r, ns, inv); break;
      case 5: any_stage<5>(tw, src, dst, n, r, ns, inv); break;
      default: any_stage<0>(tw, src, dst, n, r, ns, inv); break;
    }
    __syncthreads();
    cpx<double>* tmp = src;
    src = dst;
    dst = tmp;
    ns *= r;
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
