// cplx.cuh -- complex values, fixed-angle rotations and in-register DFTs.
//
// Two arithmetic forms share one FFT skeleton:
//   double : plain complex multiplies (the FP64 form);
//   float  : every fixed-angle rotation (FFT twiddles, e^{-iV dt}, e^{-iT dt})
//            is a three-shear lifting rotation and the radix-3 butterfly is
//            the unitary DFT3 factored into three lifting rotations.  A plain
//            FP32 complex multiply by a fixed unit phase followed later by its
//            conjugate loses ~1e-7 of norm per pair (rounding is biased for a
//            fixed angle); lifting rotations are unbiased, so FP32 errors
//            random-walk instead of drifting linearly over thousands of steps.
//
// Forward transforms use exp(+2 pi i n k / N), the sign of the reference's
// Singleton FFT with ISN = +1 (fft3d.f, called with ISN=1 in spofft.f:145).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#ifndef ESPEC_HD
#define ESPEC_HD __host__ __device__ __forceinline__
#endif

#include "rot_consts.cuh"

namespace espec {

template <typename R>
struct cpx {
  R x, y;
};

template <typename R>
ESPEC_HD cpx<R> mk(R a, R b) {
  cpx<R> c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename R>
ESPEC_HD cpx<R> operator+(cpx<R> a, cpx<R> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename R>
ESPEC_HD cpx<R> operator-(cpx<R> a, cpx<R> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename R>
ESPEC_HD cpx<R> mul_i(cpx<R> a) { return mk(-a.y, a.x); }        // * (+i)
template <typename R>
ESPEC_HD cpx<R> mul_mi(cpx<R> a) { return mk(a.y, -a.x); }       // * (-i)
template <typename R>
ESPEC_HD cpx<R> neg(cpx<R> a) { return mk(-a.x, -a.y); }
template <typename R>
ESPEC_HD cpx<R> conjg(cpx<R> a) { return mk(a.x, -a.y); }

// ---------------------------------------------------------------------------
// Rotation by a fixed angle phi (multiplication by e^{i phi}).
// ---------------------------------------------------------------------------
// FP64: stored as (cos, sin).
struct RotD {
  double c, s;
};
// FP32: stored as lifting parameters of phi' = phi - pi*[|phi| > pi/2]*sgn(phi):
// t = tan(phi'/2), s = sin(phi'), g = -1 when the pi was removed (exact negation).
struct RotF {
  float t, s, g;
};

ESPEC_HD RotD make_rotd(double phi) {
  RotD r;
#ifdef __CUDA_ARCH__
  sincos(phi, &r.s, &r.c);
#else
  r.s = sin(phi);
  r.c = cos(phi);
#endif
  return r;
}

ESPEC_HD double wrap_pi(double phi) {
  // reduce to (-pi, pi] with one FP64 remainder
  const double twopi = 6.283185307179586476925287;
  double r = remainder(phi, twopi);
  if (r <= -3.141592653589793238462643) r += twopi;
  return r;
}

ESPEC_HD RotF make_rotf(double phi) {
  const double pi = 3.141592653589793238462643;
  double p = wrap_pi(phi);
  float g = 1.0f;
  if (p > 0.5 * pi) {
    p -= pi;
    g = -1.0f;
  } else if (p < -0.5 * pi) {
    p += pi;
    g = -1.0f;
  }
  RotF r;
  r.t = (float)tan(0.5 * p);
  r.s = (float)sin(p);
  r.g = g;
  return r;
}

// apply e^{i phi}; Inv selects e^{-i phi}
template <bool Inv>
ESPEC_HD cpx<double> rot(const RotD& r, cpx<double> a) {
  const double s = Inv ? -r.s : r.s;
  return mk(fma(a.x, r.c, -a.y * s), fma(a.x, s, a.y * r.c));
}
template <bool Inv>
ESPEC_HD cpx<float> rot(const RotF& r, cpx<float> a) {
  // shears x -= t y ; y += s x ; x -= t y  (exact inverse: same with -t, -s)
  const float t = Inv ? -r.t : r.t;
  const float s = Inv ? -r.s : r.s;
  float x = a.x * r.g, y = a.y * r.g;
  x = fmaf(-t, y, x);
  y = fmaf(s, x, y);
  x = fmaf(-t, y, x);
  return mk(x, y);
}

// rotation by K*2pi/RR with K, RR compile-time (+ sign = forward), from the
// literal constants of rot_consts.cuh (multiples of 2pi/48)
template <typename R>
struct ConstRot;
template <>
struct ConstRot<double> {
  template <int J>
  static ESPEC_HD RotD get() {
    RotD r;
    r.c = rc::cd(J);
    r.s = rc::sd(J);
    return r;
  }
};
template <>
struct ConstRot<float> {
  template <int J>
  static ESPEC_HD RotF get() {
    RotF r;
    r.t = rc::tf(J);
    r.s = rc::sf(J);
    r.g = rc::gf(J);
    return r;
  }
};

template <typename R, int K, int RR, bool Inv>
ESPEC_HD cpx<R> twid_const(cpx<R> a) {
  constexpr int k = ((K % RR) + RR) % RR;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (4 * k == RR) {
    return Inv ? mul_mi(a) : mul_i(a);
  } else if constexpr (2 * k == RR) {
    return neg(a);
  } else if constexpr (4 * k == 3 * RR) {
    return Inv ? mul_i(a) : mul_mi(a);
  } else {
    static_assert((48 * k) % RR == 0, "angle not a multiple of 2pi/48");
    return rot<Inv>(ConstRot<R>::template get<(48 * k) / RR>(), a);
  }
}

// ---------------------------------------------------------------------------
// In-register DFTs, natural order in and out.  Forward: y_k = sum x_n e^{+2pi i nk/R}.
// Inv = true computes the conjugate transform (unnormalised).
// ---------------------------------------------------------------------------
template <typename R, bool Inv>
ESPEC_HD void dft2(cpx<R>* v) {
  cpx<R> a = v[0], b = v[1];
  v[0] = a + b;
  v[1] = a - b;
}

template <typename R, bool Inv>
ESPEC_HD void dft4(cpx<R>* v) {
  cpx<R> t0 = v[0] + v[2], t1 = v[0] - v[2];
  cpx<R> t2 = v[1] + v[3], t3 = v[1] - v[3];
  cpx<R> it3 = Inv ? mul_mi(t3) : mul_i(t3);
  v[0] = t0 + t2;
  v[1] = t1 + it3;
  v[2] = t0 - t2;
  v[3] = t1 - it3;
}

// DFT8 = 2 x DFT4 (even/odd) + twiddles + radix-2 butterflies; the
// conjugate transform mirrors the forward sequence (see dft12).
template <typename R, bool Inv>
ESPEC_HD void dft8(cpx<R>* v) {
  cpx<R> e[4], o[4];
  if constexpr (!Inv) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      e[k] = v[2 * k];
      o[k] = v[2 * k + 1];
    }
    dft4<R, false>(e);
    dft4<R, false>(o);
    o[1] = twid_const<R, 1, 8, false>(o[1]);
    o[2] = twid_const<R, 2, 8, false>(o[2]);
    o[3] = twid_const<R, 3, 8, false>(o[3]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = e[k] + o[k];
      v[k + 4] = e[k] - o[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      e[k] = v[k] + v[k + 4];
      o[k] = v[k] - v[k + 4];
    }
    o[1] = twid_const<R, 1, 8, true>(o[1]);
    o[2] = twid_const<R, 2, 8, true>(o[2]);
    o[3] = twid_const<R, 3, 8, true>(o[3]);
    dft4<R, true>(e);
    dft4<R, true>(o);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[2 * k] = e[k];
      v[2 * k + 1] = o[k];
    }
  }
}

template <typename R, bool Inv>
ESPEC_HD void dft16(cpx<R>* v) {
  cpx<R> e[8], o[8];
  if constexpr (!Inv) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      e[k] = v[2 * k];
      o[k] = v[2 * k + 1];
    }
    dft8<R, false>(e);
    dft8<R, false>(o);
    o[1] = twid_const<R, 1, 16, false>(o[1]);
    o[2] = twid_const<R, 2, 16, false>(o[2]);
    o[3] = twid_const<R, 3, 16, false>(o[3]);
    o[4] = twid_const<R, 4, 16, false>(o[4]);
    o[5] = twid_const<R, 5, 16, false>(o[5]);
    o[6] = twid_const<R, 6, 16, false>(o[6]);
    o[7] = twid_const<R, 7, 16, false>(o[7]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      v[k] = e[k] + o[k];
      v[k + 8] = e[k] - o[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      e[k] = v[k] + v[k + 8];
      o[k] = v[k] - v[k + 8];
    }
    o[1] = twid_const<R, 1, 16, true>(o[1]);
    o[2] = twid_const<R, 2, 16, true>(o[2]);
    o[3] = twid_const<R, 3, 16, true>(o[3]);
    o[4] = twid_const<R, 4, 16, true>(o[4]);
    o[5] = twid_const<R, 5, 16, true>(o[5]);
    o[6] = twid_const<R, 6, 16, true>(o[6]);
    o[7] = twid_const<R, 7, 16, true>(o[7]);
    dft8<R, true>(e);
    dft8<R, true>(o);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      v[2 * k] = e[k];
      v[2 * k + 1] = o[k];
    }
  }
}

// DFT3.  FP64: the textbook butterfly (gain sqrt(3) in norm).  FP32: the
// unitary DFT3/sqrt(3) written as three real lifting rotations:
//   (b, c) -> (p, m) = ((b+c), (b-c))/sqrt2          rotation by -pi/4 (+ sign)
//   (a, p) -> (y0, q)                                 rotation by -atan(sqrt 2)
//   (q, m') -> (y1, y2), m' = +i m (forward)          rotation by -pi/4 (+ sign)
template <typename R, bool Inv>
struct Dft3;

template <bool Inv>
struct Dft3<double, Inv> {
  static constexpr bool unitary = false;
  static ESPEC_HD void run(cpx<double>* v) {
    const double h = 0.8660254037844386467637232;  // sqrt(3)/2
    cpx<double> p = v[1] + v[2], m = v[1] - v[2];
    cpx<double> y0 = v[0] + p;
    cpx<double> t = mk(fma(-0.5, p.x, v[0].x), fma(-0.5, p.y, v[0].y));
    cpx<double> u = mk(h * m.x, h * m.y);
    cpx<double> iu = Inv ? mul_mi(u) : mul_i(u);
    v[0] = y0;
    v[1] = t + iu;
    v[2] = t - iu;
  }
};

ESPEC_HD void lift2(float& x, float& y, float t, float s) {
  x = fmaf(-t, y, x);
  y = fmaf(s, x, y);
  x = fmaf(-t, y, x);
}

template <bool Inv>
struct Dft3<float, Inv> {
  static constexpr bool unitary = true;
  // lifting constants of -pi/4 and -atan(sqrt(2))
  static constexpr float t45 = -0.41421356237309503f, s45 = -0.70710678118654752f;
  static constexpr float tph = -0.51763809020504152f, sph = -0.81649658092772603f;
  static ESPEC_HD void run(cpx<float>* v) {
    if constexpr (!Inv) {
      cpx<float> a = v[0], b = v[1], c = v[2];
      // (p, m): rotate (b, c) by -45deg -> ((b+c)/s2, (c-b)/s2); m = -(second)
      float px = b.x, mx = c.x, py = b.y, my = c.y;
      lift2(px, mx, t45, s45);
      lift2(py, my, t45, s45);
      mx = -mx;
      my = -my;
      // (y0, q): rotate (a, p) by -phi -> (cos a + sin p, -sin a + cos p); q = -(second)
      float y0x = a.x, qx = px, y0y = a.y, qy = py;
      lift2(y0x, qx, tph, sph);
      lift2(y0y, qy, tph, sph);
      qx = -qx;
      qy = -qy;
      // m' = +i m
      const float m2x = -my, m2y = mx;
      // (y1, y2) = ((q + m')/s2, (q - m')/s2): rotate (q, m') by -45deg, y2 = -(second)
      float y1x = qx, y2x = m2x, y1y = qy, y2y = m2y;
      lift2(y1x, y2x, t45, s45);
      lift2(y1y, y2y, t45, s45);
      v[0] = mk(y0x, y0y);
      v[1] = mk(y1x, y1y);
      v[2] = mk(-y2x, -y2y);
    } else {
      // exact mirror of the forward sequence: every lifting step undone in
      // reverse order (shears with -t, -s), so that inverse(forward(x)) = x
      // up to rounding for the rounded constants too
      float y1x = v[1].x, y1y = v[1].y, y2x = -v[2].x, y2y = -v[2].y;
      lift2(y1x, y2x, -t45, -s45);
      lift2(y1y, y2y, -t45, -s45);
      const float qx = y1x, qy = y1y, m2x = y2x, m2y = y2y;
      // m = -i m'
      float mx = m2y, my = -m2x;
      float y0x = v[0].x, y0y = v[0].y, qxx = -qx, qyy = -qy;
      lift2(y0x, qxx, -tph, -sph);
      lift2(y0y, qyy, -tph, -sph);
      const float ax = y0x, ay = y0y, px = qxx, py = qyy;
      mx = -mx;
      my = -my;
      float bx = px, cx = mx, by = py, cy = my;
      lift2(bx, cx, -t45, -s45);
      lift2(by, cy, -t45, -s45);
      v[0] = mk(ax, ay);
      v[1] = mk(bx, by);
      v[2] = mk(cx, cy);
    }
  }
};

// DFT12 = DFT4 (inner) x DFT3 (outer), n = 3 n1 + n2, k = k1 + 4 k2,
// internal twiddles exp(+2 pi i n2 k1 / 12).  The conjugate transform is the
// exact mirror of the forward sequence (DFT3^-1, inverse twiddles, conjugate
// DFT4), so that with rounded lifting constants the pair still composes to a
// multiple of the identity; the conjugate algorithm run in forward order
// leaves an O(eps) non-unitary residue that accumulates step after step.
template <typename R, bool Inv>
ESPEC_HD void dft12(cpx<R>* v) {
  cpx<R> a[3][4];
  if constexpr (!Inv) {
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < 4; ++n1) a[n2][n1] = v[3 * n1 + n2];
      dft4<R, false>(a[n2]);
    }
    a[1][1] = twid_const<R, 1, 12, false>(a[1][1]);
    a[1][2] = twid_const<R, 2, 12, false>(a[1][2]);
    a[1][3] = twid_const<R, 3, 12, false>(a[1][3]);
    a[2][1] = twid_const<R, 2, 12, false>(a[2][1]);
    a[2][2] = twid_const<R, 4, 12, false>(a[2][2]);
    a[2][3] = twid_const<R, 6, 12, false>(a[2][3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      cpx<R> b[3] = {a[0][k1], a[1][k1], a[2][k1]};
      Dft3<R, false>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) v[k1 + 4 * k2] = b[k2];
    }
  } else {
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      cpx<R> b[3] = {v[k1], v[k1 + 4], v[k1 + 8]};
      Dft3<R, true>::run(b);
#pragma unroll
      for (int n2 = 0; n2 < 3; ++n2) a[n2][k1] = b[n2];
    }
    a[1][1] = twid_const<R, 1, 12, true>(a[1][1]);
    a[1][2] = twid_const<R, 2, 12, true>(a[1][2]);
    a[1][3] = twid_const<R, 3, 12, true>(a[1][3]);
    a[2][1] = twid_const<R, 2, 12, true>(a[2][1]);
    a[2][2] = twid_const<R, 4, 12, true>(a[2][2]);
    a[2][3] = twid_const<R, 6, 12, true>(a[2][3]);
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
      dft4<R, true>(a[n2]);
#pragma unroll
      for (int n1 = 0; n1 < 4; ++n1) v[3 * n1 + n2] = a[n2][n1];
    }
  }
}

template <typename R, int RR, bool Inv>
ESPEC_HD void dft(cpx<R>* v) {
  if constexpr (RR == 2) dft2<R, Inv>(v);
  else if constexpr (RR == 3) Dft3<R, Inv>::run(v);
  else if constexpr (RR == 4) dft4<R, Inv>(v);
  else if constexpr (RR == 8) dft8<R, Inv>(v);
  else if constexpr (RR == 12) dft12<R, Inv>(v);
  else if constexpr (RR == 16) dft16<R, Inv>(v);
  else static_assert(RR == 2, "unsupported radix");
}

// norm gain^2 of one forward+conjugate pair of a radix-RR butterfly
template <typename R, int RR>
struct RadixGain {
  static constexpr int value = (RR % 3 == 0 && Dft3<R, false>::unitary) ? RR / 3 : RR;
};

}  // namespace espec
