// sod1d.cuh -- persistent batched 1D second-order-differences propagation
// with the kinetic term by FFT (eSPec's .PFSOD: psodfft.f:77-206,
// sodfft.f:64-126), FP64.
//
// One CTA owns one packet for the whole time loop; psi(t-dt) and psi(t) stay
// in registers.  Per step
//
//   psi(t+dt) = psi(t-dt) - i CST (V psi(t) + T psi(t))        [+ CST VABC psi(t)]
//
// with CST = 2 dt (au) and T psi = F^-1 (TC/N . F psi) computed by the same
// register/shared-memory FFT as the split-operator kernel (the fftshift
// swaps of sodfft.f:94-101 cancel exactly).  The first step is the
// reference's start-up: two half-size steps from psi(0) (psodfft.f:120-123).
#pragma once
#include "spo1d.cuh"

namespace espec {

struct SodTables {
  const double* vc;       // CST * V (x order)
  const double* kc;       // CST * TC / N (final FFT layout)
  const double* ab;       // CST * VABC (.VOPTIC) or mask (.SMOOTHW), x order
  const cpx<double>* w;   // conj(psi0) (x order)
};

struct SodArgs {
  SodTables tab;
  const SpoPacket* pk;
  const double2* psi0;
  const double2* psi_start;       // resume: psi(t) ...
  const double2* psi_prev_start;  // ... and psi(t - dt); no start-up step, C(0) not written
  double2* psi_out;       // psi(TF)
  double2* psi_prev_out;  // psi(TF - dt)
  double2* c_out;
  int nsteps;             // start-up step + nsteps-1 leapfrog steps
};

// kAbs: 0 none, 1 complex absorbing potential, 2 multiplicative mask
template <class PL, int kAbs>
__global__ void __launch_bounds__(PL::T) sod1d_kernel(SodArgs a) {
  using R = double;
  constexpr int N = PL::N, P = PL::P, T = PL::T;
  constexpr int NW = (T + 31) / 32;
  using Th = SpoThread<R, PL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<R>* bufs = reinterpret_cast<cpx<R>*>(smem_raw);
  double2* cpart = reinterpret_cast<double2*>(bufs + Th::NBUF * N);  // [2][NW]
  // per-point tables, structure of arrays [slot][thread]
  double* s_vc = reinterpret_cast<double*>(cpart + 2 * NW);
  double* s_kc = s_vc + N;
  double* s_ab = s_kc + N;
  cpx<R>* s_w = reinterpret_cast<cpx<R>*>(s_ab + N);

  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  const SpoPacket pk = a.pk[blockIdx.x];
  const int base = pk.off;
  double2* cout = a.c_out + pk.c_off;

  Th th;
  th.init_twiddles(t);

  cpx<R> cur[P], prev[P], wk[P];
  double c0 = 0.0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int x = base + Th::x_pos(t, j);
    const double2 p0 = a.psi_start ? a.psi_start[x] : a.psi0[x];
    cur[j] = mk(p0.x, p0.y);
    if (a.psi_start) {
      const double2 q = a.psi_prev_start[x];
      prev[j] = mk(q.x, q.y);
    } else {
      prev[j] = cur[j];
    }
    c0 += p0.x * p0.x + p0.y * p0.y;
    s_vc[j * T + t] = a.tab.vc[x];
    s_kc[j * T + t] = a.tab.kc[base + Th::final_pos(t, j)];
    if constexpr (kAbs != 0) s_ab[j * T + t] = a.tab.ab[x];
    s_w[j * T + t] = a.tab.w[x];
  }
  // C(0) (not for a resumed run)
  if (!a.psi_start) {
    double cr = c0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cr += __shfl_xor_sync(0xffffffffu, cr, o);
    if (lane == 0) cpart[warp] = make_double2(cr, 0.0);
    __syncthreads();
    if (t == 0) {
      double sr = 0.0;
      for (int i = 0; i < NW; ++i) sr += cpart[i].x;
      cout[0] = make_double2(sr, 0.0);
    }
    __syncthreads();
  }

  // dst <- dst - i f (V src + T src) [+ f ab src], dst holding the older state;
  // f = 1 (leapfrog) or 1/2 (start-up)
  auto sod_update = [&](const cpx<R>* src, cpx<R>* dst, double f) {
#pragma unroll
    for (int j = 0; j < P; ++j) wk[j] = src[j];
    th.template forward<0>(wk, bufs, t);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const double k = s_kc[j * T + t];
      wk[j] = mk(wk[j].x * k, wk[j].y * k);
    }
    th.template inverse<PL::S - 1>(wk, bufs, t);
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const double vc = s_vc[j * T + t];
      // h = vc src + T src ; dst - i f h = (dst.x + f h.y, dst.y - f h.x)
      const double hx = fma(vc, src[j].x, wk[j].x), hy = fma(vc, src[j].y, wk[j].y);
      double ox = fma(f, hy, dst[j].x), oy = fma(-f, hx, dst[j].y);
      if constexpr (kAbs == 1) {  // + f CST VABC src (sodfft.f:68-70)
        const double ab = f * s_ab[j * T + t];
        ox = fma(ab, src[j].x, ox);
        oy = fma(ab, src[j].y, oy);
      }
      if constexpr (kAbs == 2) {
        const double m = s_ab[j * T + t];
        ox *= m;
        oy *= m;
      }
      dst[j] = mk(ox, oy);
    }
  };
  // C(step) = sum conj(psi0) psi in FP64, reduced over the CTA
  auto c_sample = [&](const cpx<R>* psi, int step) {
    double cr = 0.0, ci = 0.0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const cpx<R> wj = s_w[j * T + t];
      cr = fma(wj.x, psi[j].x, fma(-wj.y, psi[j].y, cr));
      ci = fma(wj.x, psi[j].y, fma(wj.y, psi[j].x, ci));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cr += __shfl_xor_sync(0xffffffffu, cr, o);
      ci += __shfl_xor_sync(0xffffffffu, ci, o);
    }
    if (lane == 0) cpart[(step & 1) * NW + warp] = make_double2(cr, ci);
    __syncthreads();
    if (t == 0) {
      double sr = 0.0, si = 0.0;
      const double2* cp = cpart + (step & 1) * NW;
      for (int i = 0; i < NW; ++i) {
        sr += cp[i].x;
        si += cp[i].y;
      }
      cout[step] = make_double2(sr, si);
    }
  };

  bool cur_newest = true;
  int step = 2;
  if (a.psi_start) {
    step = 1;  // resumed: every step is a leapfrog step
  } else if (a.nsteps >= 1) {
    // start-up (psodfft.f:120-152): E = psi0 - i/2 H psi0 ; psi1 = psi0 - i/2 H E ;
    // then the older state is psi0 again
    sod_update(cur, prev, 0.5);  // prev = E
    sod_update(prev, cur, 0.5);  // cur = psi1
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const double2 p0 = a.psi0[base + Th::x_pos(t, j)];
      prev[j] = mk(p0.x, p0.y);
    }
    c_sample(cur, 1);
  }
  for (; step + 1 <= a.nsteps; step += 2) {  // two leapfrog steps, roles alternate
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
    const cpx<R>* nw = cur_newest ? cur : prev;
    const cpx<R>* od = cur_newest ? prev : cur;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int x = base + Th::x_pos(t, j);
      a.psi_out[x] = make_double2(nw[j].x, nw[j].y);
      if (a.psi_prev_out) a.psi_prev_out[x] = make_double2(od[j].x, od[j].y);
    }
  }
}

template <class PL>
constexpr size_t sod1d_smem_bytes() {
  using Th = SpoThread<double, PL>;
  return Th::NBUF * sizeof(cpx<double>) * PL::N + 2 * sizeof(double2) * ((PL::T + 31) / 32) +
         (size_t)PL::N * (3 * sizeof(double) + sizeof(cpx<double>));
}

}  // namespace espec
