// espec_oracle.cpp -- CPU FP64 restatement of eSPec's propagation path.
//
// TEST INFRASTRUCTURE ONLY (see espec_oracle.h).  Each function cites the
// Fortran routine of the reference (path:line under the reference's src/)
// whose arithmetic it follows.  Index arithmetic is 0-based here; the
// Fortran is 1-based.
#include "espec_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <atomic>
#include <thread>

typedef std::complex<double> cd;

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

// Fortran DO with a REAL*8 control variable: trip count max(0, INT((m2-m1+m3)/m3))
// (used by pspofft.f:110, psodfft.f:154, plnz.f:109).
extern "C" int orc_do_count(double a, double b, double c) {
  double t = (b - a + c) / c;
  if (!(t > 0.0)) return 0;
  return (int)t;  // INT truncates toward zero
}

// fcorrel.f:60-65  plain left-to-right real dot product
extern "C" double orc_fcorrel(int n, const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// ecnorm.f:59-65  2-norm
extern "C" double orc_ecnorm(int n, const double* a) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * a[i];
  return std::sqrt(s);
}

// ---------------------------------------------------------------------------
// FFT.  The reference uses Singleton's 1968 mixed-radix FFT (fft3d.f:1-606),
// one call per variable of a column-major multi-dimensional array.  Any
// exact DFT is arithmetically equivalent up to rounding; this is a recursive
// mixed-radix Cooley-Tukey with per-length cached twiddle tables.  isn > 0
// selects exp(+2 pi i jk/n), isn < 0 exp(-2 pi i jk/n); unnormalised.
// ---------------------------------------------------------------------------
namespace {

// Plan of an iterative Stockham autosort FFT of length n: radices in
// execution order and, per stage, the twiddles exp(+2 pi i j k / (l r)).
struct FftPlan {
  int n = 0;
  std::vector<int> radix;
  std::vector<std::vector<cd>> tw;  // per stage: tw[k*(r) + j]
};

std::vector<int> factorise(int n) {
  std::vector<int> f;
  while (n % 4 == 0) {
    f.push_back(4);
    n /= 4;
  }
  while (n % 2 == 0) {
    f.push_back(2);
    n /= 2;
  }
  for (int p = 3; n > 1; p += 2)
    while (n % p == 0) {
      f.push_back(p);
      n /= p;
    }
  return f;
}

const FftPlan& fft_plan(int n) {
  static std::mutex mu;
  static std::map<int, FftPlan*> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(n);
  if (it != cache.end()) return *it->second;
  FftPlan* pl = new FftPlan;
  pl->n = n;
  pl->radix = factorise(n);
  int l = 1;  // product of the radices already applied
  for (int r : pl->radix) {
    const int m = n / (l * r);
    (void)m;
    std::vector<cd> w((size_t)l * r);
    for (int k = 0; k < l; ++k)
      for (int j = 0; j < r; ++j) {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)(j * k) /
                        (long double)(l * r);
        w[(size_t)k * r + j] = cd((double)cosl(a), (double)sinl(a));
      }
    pl->tw.push_back(std::move(w));
    l *= r;
  }
  cache[n] = pl;
  return *pl;
}

// one Stockham pass: x (length n, viewed as [r][m][l] with m = n/(l r)) ->
// y viewed as [m][r][l]; sub-transforms of length l*r.
void stockham_pass(const cd* x, cd* y, int n, int l, int r, const cd* tw, int sign) {
  const int m = n / (l * r);
  cd tmp[16];
  std::vector<cd> big;
  cd* t = tmp;
  if (r > 16) {
    big.resize(r);
    t = big.data();
  }
  for (int q = 0; q < m; ++q) {
    for (int k = 0; k < l; ++k) {
      // gather the r inputs of this butterfly, apply twiddles
      for (int j = 0; j < r; ++j) {
        cd v = x[(size_t)j * m * l + (size_t)q * l + k];
        if (k && j) {
          const cd w = tw[(size_t)k * r + j];
          const double wi = sign > 0 ? w.imag() : -w.imag();
          v = cd(v.real() * w.real() - v.imag() * wi, v.real() * wi + v.imag() * w.real());
        }
        t[j] = v;
      }
      cd* out = const_cast<cd*>(y) + (size_t)q * r * l + k;
      if (r == 2) {
        out[0] = t[0] + t[1];
        out[l] = t[0] - t[1];
      } else if (r == 4) {
        cd a0 = t[0] + t[2], a1 = t[0] - t[2], b0 = t[1] + t[3], b1 = t[1] - t[3];
        cd jb = sign > 0 ? cd(-b1.imag(), b1.real()) : cd(b1.imag(), -b1.real());
        out[0] = a0 + b0;
        out[l] = a1 + jb;
        out[2 * l] = a0 - b0;
        out[3 * l] = a1 - jb;
      } else if (r == 3) {
        const double h = 0.8660254037844386467637232;  // sqrt(3)/2
        cd p = t[1] + t[2], mm = t[1] - t[2];
        cd c = cd(t[0].real() - 0.5 * p.real(), t[0].imag() - 0.5 * p.imag());
        cd u = cd(h * mm.real(), h * mm.imag());
        cd iu = sign > 0 ? cd(-u.imag(), u.real()) : cd(u.imag(), -u.real());
        out[0] = t[0] + p;
        out[l] = c + iu;
        out[2 * l] = c - iu;
      } else {
        // generic odd radix: W_r^{js} from the stage table (entry k = l/.. unused)
        for (int s2 = 0; s2 < r; ++s2) {
          double ar = 0.0, ai = 0.0;
          for (int j = 0; j < r; ++j) {
            const double ang = 6.283185307179586476925287 * (double)((j * s2) % r) / (double)r;
            const double c = std::cos(ang), sn = sign > 0 ? std::sin(ang) : -std::sin(ang);
            ar += t[j].real() * c - t[j].imag() * sn;
            ai += t[j].real() * sn + t[j].imag() * c;
          }
          out[(size_t)s2 * l] = cd(ar, ai);
        }
      }
    }
  }
}

// unnormalised DFT of x in place: sign > 0 -> exp(+2 pi i jk/n)
void dft_line(cd* x, int n, int sign) {
  // per-thread memo of the last plan: the shared cache's lock is taken once
  // per length and thread, not once per line (host threads of the batched
  // CPU runs would otherwise contend on it every step)
  thread_local int memo_n = 0;
  thread_local const FftPlan* memo = nullptr;
  if (memo_n != n) {
    memo = &fft_plan(n);
    memo_n = n;
  }
  const FftPlan& pl = *memo;
  thread_local std::vector<cd> buf;
  if ((int)buf.size() < n) buf.resize(n);
  cd* a = x;
  cd* b = buf.data();
  int l = 1;
  for (size_t s = 0; s < pl.radix.size(); ++s) {
    const int r = pl.radix[s];
    stockham_pass(a, b, n, l, r, pl.tw[s].data(), sign);
    std::swap(a, b);
    l *= r;
  }
  if (a != x)
    for (int i = 0; i < n; ++i) x[i] = a[i];
}

}  // namespace

// Singleton interface: ntot values, variable of length n, nspan = n * (stride)
extern "C" void orc_fft(double* re, double* im, int ntot, int n, int nspan, int isn) {
  if (n < 2) return;
  const int stride = nspan / n;
  const int sign = isn >= 0 ? +1 : -1;
  thread_local std::vector<cd> line;
  if ((int)line.size() < n) line.resize(n);
  for (int base = 0; base < ntot; base += nspan) {
    for (int off = 0; off < stride; ++off) {
      for (int j = 0; j < n; ++j) {
        int idx = base + off + j * stride;
        line[j] = cd(re[idx], im[idx]);
      }
      dft_line(line.data(), n, sign);
      for (int j = 0; j < n; ++j) {
        int idx = base + off + j * stride;
        re[idx] = line[j].real();
        im[idx] = line[j].imag();
      }
    }
  }
}

static void fft_all_axes(int ndim, const int* np, int n, double* re, double* im, int isn) {
  int nf = 1;
  for (int i = 0; i < ndim; ++i) {  // spofft.f:142-146
    nf *= np[i];
    orc_fft(re, im, n, np[i], nf, isn);
  }
}

// ---------------------------------------------------------------------------
// dkeft.f:64-137  DIGT kinetic table in FFT order.
// ---------------------------------------------------------------------------
static const double DIGT_TWOPI = 6.283185307;  // dkeft.f:38 (truncated literal)

static void digt_axis(int np, double sh, double sm, double* t) {
  // dkeft.f:69-79: P accumulated by repeated addition
  const double dp = DIGT_TWOPI / (np * sh);
  double p = 0.0;
  for (int i = 0; i < np / 2; ++i) {
    t[i] = p * p / (2.0 * sm);
    p = p + dp;
  }
  p = -p;
  for (int i = np / 2; i < np; ++i) {
    t[i] = p * p / (2.0 * sm);
    p = p + dp;
  }
}

extern "C" void orc_digt(int ndim, const int* np, const double* sh, const double* sm,
                         double* tc, double* b, int quirks) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  *b = 1.0 / n;  // dkeft.f:66,82,106
  if (ndim == 1) {
    digt_axis(np[0], sh[0], sm[0], tc);
    return;
  }
  if (quirks & ORC_Q_DIGT_ND) {
    // literal 2D/3D loops of dkeft.f:80-137: only TC(1..NP1) is written
    for (int i = 0; i < n; ++i) tc[i] = 0.0;
    double dp[3];
    for (int a = 0; a < ndim; ++a) dp[a] = DIGT_TWOPI / (np[a] * sh[a]);
    if (ndim == 2) {
      double p1 = 0, p2 = 0;
      for (int j = 0; j < np[1] / 2; ++j) {
        for (int i = 0; i < np[0] / 2; ++i) {
          tc[i] = p1 * p1 / (2 * sm[0]) + p2 * p2 / (2 * sm[1]);
          p1 = p1 + dp[0];
        }
        p2 = p2 + dp[1];
      }
      p1 = -(p1 + dp[0]);
      p2 = -(p2 + dp[1]);
      for (int j = np[1] / 2; j < np[1]; ++j) {
        for (int i = np[0] / 2; i < np[0]; ++i) {
          tc[i] = p1 * p1 / (2 * sm[0]) + p2 * p2 / (2 * sm[1]);
          p1 = p1 + dp[0];
        }
        p2 = p2 + dp[1];
      }
    } else {
      double p1 = 0, p2 = 0, p3 = 0;
      for (int k = 0; k < np[2] / 2; ++k) {
        for (int j = 0; j < np[1] / 2; ++j) {
          for (int i = 0; i < np[0] / 2; ++i) {
            tc[i] = p1 * p1 / (2 * sm[0]) + p2 * p2 / (2 * sm[1]) + p3 * p3 / (2 * sm[2]);
            p1 = p1 + dp[0];
          }
          p2 = p2 + dp[1];
        }
        p3 = p3 + dp[2];
      }
      p1 = -(p1 + dp[0]);
      p2 = -(p2 + dp[1]);
      p3 = -(p3 + dp[2]);
      // dkeft.f:127-137 loops J and I start at NP/2 (not NP/2+1)
      for (int k = np[2] / 2; k < np[2]; ++k) {
        for (int j = np[1] / 2 - 1; j < np[1]; ++j) {
          for (int i = np[0] / 2 - 1; i < np[0]; ++i) {
            tc[i] = p1 * p1 / (2 * sm[0]) + p2 * p2 / (2 * sm[1]) + p3 * p3 / (2 * sm[2]);
            p1 = p1 + dp[0];
          }
          p2 = p2 + dp[1];
        }
        p3 = p3 + dp[2];
      }
    }
    return;
  }
  // corrected N-D table: outer sum of the per-axis 1D tables
  std::vector<double> t[3];
  for (int a = 0; a < ndim; ++a) {
    t[a].resize(np[a]);
    digt_axis(np[a], sh[a], sm[a], t[a].data());
  }
  if (ndim == 2) {
    for (int j = 0; j < np[1]; ++j)
      for (int i = 0; i < np[0]; ++i) tc[i + np[0] * j] = t[0][i] + t[1][j];
  } else {
    for (int k = 0; k < np[2]; ++k)
      for (int j = 0; j < np[1]; ++j)
        for (int i = 0; i < np[0]; ++i)
          tc[i + np[0] * (j + np[1] * k)] = t[0][i] + t[1][j] + t[2][k];
  }
}

// ---------------------------------------------------------------------------
// au1d.f:52-73, au2di.f:57-225, au3d.f:61-117: H_FD u with the 5-point
// 4th-order stencil SHM*(1,-16,30,-16,1) per axis plus V u; values outside
// the grid are zero.
// ---------------------------------------------------------------------------
extern "C" void orc_au(int ndim, const int* np, const double* shm, const double* vpot,
                       const double* u, double* out) {
  const int nx = np[0], ny = ndim > 1 ? np[1] : 1, nz = ndim > 2 ? np[2] : 1;
  double sht = 0.0;
  for (int a = 0; a < ndim; ++a) sht += shm[a];
  const long sx = 1, sy = nx, sz = (long)nx * ny;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long c = i + sy * j + sz * k;
        double s = (30.0 * sht + vpot[c]) * u[c];
        const int idx[3] = {i, j, k};
        const int len[3] = {nx, ny, nz};
        const long str[3] = {sx, sy, sz};
        for (int a = 0; a < ndim; ++a) {
          const double h = shm[a];
          if (idx[a] >= 2) s += h * u[c - 2 * str[a]];
          if (idx[a] >= 1) s += -16.0 * h * u[c - str[a]];
          if (idx[a] + 1 < len[a]) s += -16.0 * h * u[c + str[a]];
          if (idx[a] + 2 < len[a]) s += h * u[c + 2 * str[a]];
        }
        out[c] = s;
      }
}

// eigenerg.f:56-66  <u|H_FD|u>
extern "C" double orc_eigenerg(int ndim, const int* np, const double* shm,
                               const double* vpot, const double* u) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  std::vector<double> w(n);
  orc_au(ndim, np, shm, vpot, u, w.data());
  return orc_fcorrel(n, u, w.data());
}

// eigenergfft.f:58-100  EFFT4 = sum V|psi|^2 + Re<psi|T_FFT|psi>
extern "C" double orc_efft4(int ndim, const int* np, double b, const double* u,
                            const double* v, const double* tc, const double* vpot) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  const int nh = n / 2;
  double su1 = 0, sv1 = 0;
  for (int i = 0; i < n; ++i) {
    su1 = su1 + u[i] * vpot[i] * u[i];
    sv1 = sv1 + v[i] * vpot[i] * v[i];
  }
  std::vector<double> wu(n), wv(n);
  for (int i = 0; i < nh; ++i) {
    wu[i] = u[i + nh];
    wv[i] = v[i + nh];
    wu[i + nh] = u[i];
    wv[i + nh] = v[i];
  }
  fft_all_axes(ndim, np, n, wu.data(), wv.data(), 1);
  for (int i = 0; i < n; ++i) {
    wu[i] = tc[i] * wu[i];
    wv[i] = tc[i] * wv[i];
  }
  fft_all_axes(ndim, np, n, wu.data(), wv.data(), -1);
  double su2 = 0, sv2 = 0;
  for (int i = 0; i < nh; ++i) {
    su2 = su2 + u[i] * b * wu[i + nh];
    sv2 = sv2 + v[i] * b * wv[i + nh];
    su2 = su2 + u[i + nh] * b * wu[i];
    sv2 = sv2 + v[i + nh] * b * wv[i];
  }
  return su1 + su2 + sv1 + sv2;
}

// ---------------------------------------------------------------------------
// spofft.f:64-200  PSPOFFTAUX: one split-operator step, in place.
// ---------------------------------------------------------------------------
extern "C" void orc_spo_step(int ndim, const int* np, double b, double cst1, double cst2,
                             const double* tc, const double* vpot, const double* vabc,
                             int absorb, int quirks, double* u, double* v) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  const int nh = n / 2;
  const bool voptic = absorb == ORC_ABS_VOPTIC;
  const bool smooth = absorb == ORC_ABS_SMOOTHW;
  // first V half-step with the half swap (spofft.f:66-81 / :120-133)
  for (int i = 0; i < nh; ++i) {
    double th1 = cst2 * vpot[i];
    double c1, s1;
    sincos(th1, &s1, &c1);
    if (voptic) {
      double e1 = std::exp(cst2 * vabc[i]);
      c1 *= e1;
      s1 *= e1;
    }
    double ua = c1 * u[i] + s1 * v[i];
    double va = c1 * v[i] - s1 * u[i];
    double th2 = cst2 * vpot[i + nh];
    double c2, s2;
    sincos(th2, &s2, &c2);
    if (voptic) {
      double e2 = std::exp(cst2 * vabc[i + nh]);
      c2 *= e2;
      s2 *= e2;
    }
    u[i] = c2 * u[i + nh] + s2 * v[i + nh];
    v[i] = c2 * v[i + nh] - s2 * u[i + nh];
    u[i + nh] = ua;
    v[i + nh] = va;
  }
  fft_all_axes(ndim, np, n, u, v, 1);
  // kinetic phase (spofft.f:148-154)
  for (int i = 0; i < n; ++i) {
    double th = cst1 * tc[i];
    double c, s;
    sincos(th, &s, &c);
    double un = c * u[i] + s * v[i];
    if (quirks & ORC_Q_SPO_INPLACE) {
      u[i] = un;
      v[i] = c * v[i] - s * u[i];  // uses the updated U(I)
    } else {
      v[i] = c * v[i] - s * u[i];
      u[i] = un;
    }
  }
  fft_all_axes(ndim, np, n, u, v, -1);
  // last V half-step with swap back and 1/N (spofft.f:103-118 / :162-191)
  for (int i = 0; i < nh; ++i) {
    double th1 = cst2 * vpot[i + nh];
    double c1, s1;
    sincos(th1, &s1, &c1);
    if (voptic) {
      double e1 = std::exp(cst2 * vabc[i + nh]);
      c1 *= e1;
      s1 *= e1;
    }
    double ua = c1 * b * u[i] + s1 * b * v[i];
    double va = c1 * b * v[i] - s1 * b * u[i];
    double th2 = cst2 * vpot[i];
    double c2, s2;
    sincos(th2, &s2, &c2);
    if (voptic) {
      double e2 = std::exp(cst2 * vabc[i]);
      c2 *= e2;
      s2 *= e2;
    }
    double un = c2 * b * u[i + nh] + s2 * b * v[i + nh];
    double vn = c2 * b * v[i + nh] - s2 * b * u[i + nh];
    if (smooth) {
      u[i] = vabc[i] * un;
      v[i] = vabc[i] * vn;
      u[i + nh] = vabc[i + nh] * ua;
      v[i + nh] = vabc[i + nh] * va;
    } else {
      u[i] = un;
      v[i] = vn;
      u[i + nh] = ua;
      v[i + nh] = va;
    }
  }
}

// sodfft.f:64-126  PSODFFTAUX: psi+ = psi- - i cst H psi (T by FFT)
static void sod_step(int ndim, const int* np, double b, double cst, const double* tc,
                     const double* vpot, const double* vabc, int absorb, int quirks,
                     double* u1, double* u2, double* v1, double* v2, double* wr, double* wi) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  const int nh = n / 2;
  if (absorb == ORC_ABS_VOPTIC) {
    for (int i = 0; i < n; ++i) {
      wr[i] = u1[i] + cst * vpot[i] * v2[i] + cst * vabc[i] * u2[i];
      wi[i] = v1[i] - cst * vpot[i] * u2[i] + cst * vabc[i] * v2[i];
      u1[i] = u2[i];
      v1[i] = v2[i];
    }
  } else {
    for (int i = 0; i < n; ++i) {
      wr[i] = u1[i] + cst * vpot[i] * v2[i];
      wi[i] = v1[i] - cst * vpot[i] * u2[i];
      u1[i] = u2[i];
      v1[i] = v2[i];
    }
  }
  for (int i = 0; i < nh; ++i) {
    double ua = u2[i], va = v2[i];
    u2[i] = u2[i + nh];
    v2[i] = v2[i + nh];
    u2[i + nh] = ua;
    v2[i + nh] = va;
  }
  fft_all_axes(ndim, np, n, u2, v2, 1);
  for (int i = 0; i < n; ++i) {
    u2[i] = tc[i] * u2[i];
    v2[i] = tc[i] * v2[i];
  }
  fft_all_axes(ndim, np, n, u2, v2, -1);
  // sodfft.f:108 tests TPABSOR(1:7) against the 8-character '.SMOOTHW', which
  // never matches: the reference never applies the mask in this propagator.
  const bool smooth = absorb == ORC_ABS_SMOOTHW && !(quirks & ORC_Q_SOD_SMOOTHW);
  for (int i = 0; i < nh; ++i) {
    double ua = wr[i + nh] + cst * b * v2[i];
    double va = wi[i + nh] - cst * b * u2[i];
    double ul = wr[i] + cst * b * v2[i + nh];
    double vl = wi[i] - cst * b * u2[i + nh];
    if (smooth) {
      u2[i] = vabc[i] * ul;
      v2[i] = vabc[i] * vl;
      u2[i + nh] = vabc[i + nh] * ua;
      v2[i + nh] = vabc[i + nh] * va;
    } else {
      u2[i] = ul;
      v2[i] = vl;
      u2[i + nh] = ua;
      v2[i + nh] = va;
    }
  }
}

// ---------------------------------------------------------------------------
// absorb.f:62-195  ABSORBINGBC
// ---------------------------------------------------------------------------
extern "C" int orc_absorbingbc(int ndim, const int* np, int type, const double* al,
                               const double* ar, const double* sh, const double* xi,
                               const double* xf, const double* voi, double* vabc) {
  if (ndim == 1) {
    for (int i = 0; i < np[0]; ++i) {
      double x1 = xi[0] + (i) * sh[0];  // XI(1) + (I - ONE)*SH(1)
      double r;
      switch (type) {
        case ORC_ABC_SMOOTHW:  // absorb.f:66-79
          if (x1 < al[0])
            r = std::exp(voi[0] * std::pow(x1 - al[0], voi[1]) / (x1 + sh[0] - xi[0]));
          else if (x1 > ar[0])
            r = std::exp(-voi[0] * (x1 - ar[0]) / std::pow(xf[0] + sh[0] - x1, voi[1]));
          else
            r = 1.0;
          break;
        case ORC_ABC_SMRS:  // absorb.f:82-118 (active lines)
          if (x1 < al[0])
            r = 1.0 - voi[0] * (x1 - al[0]) * (x1 - al[0]);
          else if (x1 > ar[0])
            r = 1.0 - voi[0] * (x1 - ar[0]) * (x1 - ar[0]);
          else
            r = 1.0;
          break;
        case ORC_ABC_VOPTIC_LINEAR:  // absorb.f:120-130
          if (x1 < al[0])
            r = -voi[0] * (x1 - al[0]) / (x1 + sh[0] - xi[0]);
          else if (x1 > ar[0])
            r = voi[0] * (x1 - ar[0]) / (xf[0] + sh[0] - x1);
          else
            r = 0.0;
          break;
        case ORC_ABC_VOPTIC_POLIN:  // absorb.f:142-152
          if (x1 < al[0])
            r = voi[0] * std::pow(x1 - al[0], voi[1]);
          else if (x1 > ar[0])
            r = voi[0] * std::pow(x1 - ar[0], voi[1]);
          else
            r = 0.0;
          break;
        default:
          return -1;
      }
      vabc[i] = r;
    }
    return 0;
  }
  if (ndim == 2 && type == ORC_ABC_SMOOTHW) {  // absorb.f:157-195
    for (int j = 0; j < np[1]; ++j) {
      double x2 = xi[1] + j * sh[1];
      for (int i = 0; i < np[0]; ++i) {
        double x1 = xi[0] + i * sh[0];
        double r;
        if (x1 < al[0])
          r = std::exp(voi[0] * (x1 - al[0]) / (x1 + sh[0] - xi[0]));
        else if (x2 < al[1])
          r = std::exp(voi[1] * (x2 - al[1]) / (x2 + sh[1] - xi[1]));
        else if (x1 > ar[0])
          r = std::exp(-voi[0] * (x1 - ar[0]) / (xf[0] + sh[0] - x1));
        else if (x2 > ar[1])
          r = std::exp(-voi[1] * (x2 - ar[1]) / (xf[1] + sh[1] - x2));
        else
          r = 1.0;
        vabc[i + np[0] * j] = r;
      }
    }
    return 0;
  }
  return -1;  // absorb.f:196-205 STOP: not implemented in the reference
}

// ---------------------------------------------------------------------------
// Propagator drivers
// ---------------------------------------------------------------------------
namespace {
struct RowSink {
  double* rows;
  int cap;
  int n = 0;
  void put(double t, double e, double cr, double ci, double ct, double fn) {
    if (rows && n < cap) {
      double* r = rows + 6 * n;
      r[0] = t;
      r[1] = e;
      r[2] = cr;
      r[3] = ci;
      r[4] = ct;
      r[5] = fn;
    }
    ++n;
  }
};
struct CSink {
  double *re, *im;
  int cap;
  int n = 0;
  void put(double cr, double ci) {
    if (n < cap) {
      re[n] = cr;
      im[n] = ci;
    }
    ++n;
  }
};
inline int npts(const orc_prop_t* p) {
  int n = 1;
  for (int a = 0; a < p->ndim; ++a) n *= p->np[a];
  return n;
}
}  // namespace

// pspofft.f:72-145  PSPOFFT
extern "C" int orc_pspofft(const orc_prop_t* p, const double* vpot, const double* vabc,
                           double* u1, double* v1, double* c_re, double* c_im, int c_cap,
                           double* rows, int row_cap, int* nrows, int* info) {
  const int n = npts(p);
  RowSink rs{rows, row_cap};
  CSink cs{c_re, c_im, c_cap};
  *info = 0;
  int mc = 0;
  double t = p->ti;
  const double cst1 = p->dt / ORC_SHFS, cst2 = p->dt / (2.0 * ORC_SHFS);
  std::vector<double> u0(u1, u1 + n), v0(v1, v1 + n), tc(n);
  double b;
  orc_digt(p->ndim, p->np, p->sh, p->sm, tc.data(), &b, p->quirks);
  auto corr = [&](double& cr, double& ci) {
    cr = orc_fcorrel(n, u0.data(), u1) + orc_fcorrel(n, v0.data(), v1);
    ci = orc_fcorrel(n, u0.data(), v1) - orc_fcorrel(n, v0.data(), u1);
  };
  auto normf = [&]() {
    double fnr = orc_fcorrel(n, u1, u1) + orc_fcorrel(n, v1, v1);
    double fni = orc_fcorrel(n, u1, v1) - orc_fcorrel(n, v1, u1);
    return std::sqrt(fnr * fnr + fni * fni);
  };
  double cr, ci;
  corr(cr, ci);
  double ct = std::sqrt(cr * cr + ci * ci);
  cs.put(cr, ci);
  double et = orc_efft4(p->ndim, p->np, b, u1, v1, tc.data(), vpot);
  const double e0 = et;
  double fnt = normf();
  const double f0 = fnt;
  if (p->prtcrl != ORC_PRT_NONE) rs.put(t, et, cr, ci, ct, fnt);
  const int nit = orc_do_count(p->ti + p->dt, p->tf + p->dt, p->dt);
  t = p->ti + p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    orc_spo_step(p->ndim, p->np, b, cst1, cst2, tc.data(), vpot, vabc, p->absorb, p->quirks,
                 u1, v1);
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      corr(cr, ci);
      cs.put(cr, ci);
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      corr(cr, ci);
      ct = std::sqrt(cr * cr + ci * ci);
      et = orc_efft4(p->ndim, p->np, b, u1, v1, tc.data(), vpot);
      fnt = normf();
      if (p->absorb != ORC_ABS_NONE) {  // pspofft.f:137-142
        if (std::fabs((et - e0) / e0) * 100.0 > p->tol ||
            std::fabs((fnt - f0) / f0) * 100.0 > p->tol)
          *info = 1;
      } else {
        if (std::fabs((et - e0) / e0) * 100.0 > p->tol) *info = 1;
      }
      rs.put(t, et, cr, ci, ct, fnt);
    }
  }
  if (nrows) *nrows = rs.n;
  return cs.n;
}

// psodfft.f:77-206  PSODFFT
extern "C" int orc_psodfft(const orc_prop_t* p, const double* vpot, const double* vabc,
                           double* u1, double* v1, double* u2, double* v2, double* c_re,
                           double* c_im, int c_cap, double* rows, int row_cap, int* nrows,
                           int* info) {
  const int n = npts(p);
  RowSink rs{rows, row_cap};
  CSink cs{c_re, c_im, c_cap};
  *info = 0;
  double t = p->ti;
  const double cst = 2.0 * p->dt / ORC_SHFS;
  std::vector<double> u0(u1, u1 + n), v0(v1, v1 + n), tc(n), wr(n), wi(n);
  for (int i = 0; i < n; ++i) {
    u2[i] = u0[i];
    v2[i] = v0[i];
  }
  double b;
  orc_digt(p->ndim, p->np, p->sh, p->sm, tc.data(), &b, p->quirks);
  auto corr = [&](double& cr, double& ci) {
    cr = orc_fcorrel(n, u0.data(), u2) + orc_fcorrel(n, v0.data(), v2);
    ci = orc_fcorrel(n, u0.data(), v2) - orc_fcorrel(n, v0.data(), u2);
  };
  auto normf = [&]() {
    double fnr = orc_fcorrel(n, u2, u2) + orc_fcorrel(n, v2, v2);
    double fni = orc_fcorrel(n, u2, v2) - orc_fcorrel(n, v2, u2);
    return std::sqrt(fnr * fnr + fni * fni);
  };
  auto drift = [&](double et, double e0, double fnt, double f0) {  // psodfft.f:178-183
    if (p->absorb != ORC_ABS_NONE) {
      if (std::fabs((et - e0) / e0) * 100.0 > p->tol) *info = 1;
    } else {
      if (std::fabs((et - e0) / e0) * 100.0 > p->tol ||
          std::fabs((fnt - f0) / f0) * 100.0 > p->tol)
        *info = 1;
    }
  };
  double cr, ci;
  corr(cr, ci);
  double ct = std::sqrt(cr * cr + ci * ci);
  cs.put(cr, ci);
  double et = orc_efft4(p->ndim, p->np, b, u2, v2, tc.data(), vpot);
  const double e0 = et;
  double fnt = normf();
  const double f0 = fnt;
  if (p->prtcrl != ORC_PRT_NONE) rs.put(t, et, cr, ci, ct, fnt);
  // start-up: two half-steps (psodfft.f:120-123)
  sod_step(p->ndim, p->np, b, cst / 2.0, tc.data(), vpot, vabc, p->absorb, p->quirks, u1, u2,
           v1, v2, wr.data(), wi.data());
  sod_step(p->ndim, p->np, b, cst / 2.0, tc.data(), vpot, vabc, p->absorb, p->quirks, u1, u2,
           v1, v2, wr.data(), wi.data());
  int mc = 1;
  t = p->ti + p->dt;
  corr(cr, ci);
  ct = std::sqrt(cr * cr + ci * ci);
  if (mc == p->lc) {
    mc = 0;
    cs.put(cr, ci);
  }
  if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
    et = orc_efft4(p->ndim, p->np, b, u2, v2, tc.data(), vpot);
    fnt = normf();
    rs.put(t, et, cr, ci, ct, fnt);
  }
  for (int i = 0; i < n; ++i) {  // psodfft.f:149-152
    u1[i] = u0[i];
    v1[i] = v0[i];
  }
  const int nit = orc_do_count(p->ti + 2 * p->dt, p->tf + p->dt, p->dt);
  t = p->ti + 2 * p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    sod_step(p->ndim, p->np, b, cst, tc.data(), vpot, vabc, p->absorb, p->quirks, u1, u2, v1,
             v2, wr.data(), wi.data());
    mc = mc + 1;
    if (mc == p->lc) {
      corr(cr, ci);
      mc = 0;
      cs.put(cr, ci);
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      corr(cr, ci);
      ct = std::sqrt(cr * cr + ci * ci);
      et = orc_efft4(p->ndim, p->np, b, u2, v2, tc.data(), vpot);
      fnt = normf();
      drift(et, e0, fnt, f0);
      rs.put(t, et, cr, ci, ct, fnt);
    }
  }
  et = orc_efft4(p->ndim, p->np, b, u2, v2, tc.data(), vpot);
  fnt = normf();
  drift(et, e0, fnt, f0);
  if (nrows) *nrows = rs.n;
  return cs.n;
}

// sod.f:64-123  PSODAUX with H = AU (4th-order finite differences):
// U2 <- U1 + cst H V2, then V2 <- V1 - cst H U2(old), the old (U2, V2) moving
// to (U1, V1); .VOPTIC subtracts cst VABC times the old value, .SMOOTHW
// multiplies the result by the mask (sod.f:71-119)
static void psod_aux(const orc_prop_t* p, double cst, const double* vpot, const double* vabc,
                     double* u1, double* u2, double* v1, double* v2, double* work) {
  const int n = npts(p);
  orc_au(p->ndim, p->np, p->shm, vpot, v2, work);
  for (int i = 0; i < n; ++i) {
    const double uaux = u2[i];
    if (p->absorb == ORC_ABS_VOPTIC)
      u2[i] = u1[i] + cst * work[i] - cst * vabc[i] * uaux;
    else if (p->absorb == ORC_ABS_SMOOTHW)
      u2[i] = vabc[i] * (u1[i] + cst * work[i]);
    else
      u2[i] = u1[i] + cst * work[i];
    u1[i] = uaux;
  }
  orc_au(p->ndim, p->np, p->shm, vpot, u1, work);
  for (int i = 0; i < n; ++i) {
    const double vaux = v2[i];
    if (p->absorb == ORC_ABS_VOPTIC)
      v2[i] = v1[i] - cst * work[i] - cst * vabc[i] * vaux;
    else if (p->absorb == ORC_ABS_SMOOTHW)
      v2[i] = vabc[i] * (v1[i] - cst * work[i]);
    else
      v2[i] = v1[i] - cst * work[i];
    v1[i] = vaux;
  }
}

// psod.f:64-205  PSOD: C(0); an Euler half step (CST/4) and a midpoint step
// (CST/2) to TI + DT; (U1, V1) back to psi0; then leapfrog steps of CST =
// 2 DT / SHFS.  Printed rows carry |C|^2 and E = EIGENERG(U) + EIGENERG(V);
// the norm column is sum |psi|^2, squared in the rows of the loop
// (psod.f:183), which the loop's drift test also uses.
extern "C" int orc_psod(const orc_prop_t* p, const double* vpot, const double* vabc, double* u1,
                        double* v1, double* u2, double* v2, double* c_re, double* c_im, int c_cap,
                        double* rows, int row_cap, int* nrows, int* info) {
  const int n = npts(p);
  RowSink rs{rows, row_cap};
  CSink cs{c_re, c_im, c_cap};
  *info = 0;
  double t = p->ti;
  const double cst = 2.0 * p->dt / ORC_SHFS;
  const bool absorb = p->absorb != ORC_ABS_NONE;
  std::vector<double> u0(u1, u1 + n), v0(v1, v1 + n), work(n);
  for (int i = 0; i < n; ++i) {
    u2[i] = u0[i];
    v2[i] = v0[i];
  }
  auto corr = [&](double& cr, double& ci) {
    cr = orc_fcorrel(n, u0.data(), u2) + orc_fcorrel(n, v0.data(), v2);
    ci = orc_fcorrel(n, u0.data(), v2) - orc_fcorrel(n, v0.data(), u2);
  };
  auto energy = [&]() {
    return orc_eigenerg(p->ndim, p->np, p->shm, vpot, u2) +
           orc_eigenerg(p->ndim, p->np, p->shm, vpot, v2);
  };
  auto norm2 = [&]() { return orc_fcorrel(n, u2, u2) + orc_fcorrel(n, v2, v2); };
  auto drifted = [&](double et, double e0, double fnt, double f0) {
    return std::fabs((et - e0) / e0) * 100.0 > p->tol || std::fabs((fnt - f0) / f0) * 100.0 > p->tol;
  };
  double cr, ci;
  corr(cr, ci);
  cs.put(cr, ci);
  double et = energy();
  const double e0 = et;
  double fnt = norm2();
  const double f0 = fnt;
  if (p->prtcrl != ORC_PRT_NONE) rs.put(t, et, cr, ci, cr * cr + ci * ci, fnt);
  psod_aux(p, cst / 4.0, vpot, vabc, u1, u2, v1, v2, work.data());
  psod_aux(p, cst / 2.0, vpot, vabc, u1, u2, v1, v2, work.data());
  int mc = 1;
  t = p->ti + p->dt;
  if (mc == p->lc) {
    mc = 0;
    corr(cr, ci);
    cs.put(cr, ci);
  }
  if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
    corr(cr, ci);
    et = energy();
    fnt = norm2();
    rs.put(t, et, cr, ci, cr * cr + ci * ci, fnt);
  }
  for (int i = 0; i < n; i += 2) {  // psod.f:136-141
    u1[i] = u0[i];
    v1[i] = v0[i];
    if (i + 1 < n) {
      u1[i + 1] = u0[i + 1];
      v1[i + 1] = (p->quirks & ORC_Q_PSOD_COPY) ? v0[i] : v0[i + 1];
    }
  }
  const int nit = orc_do_count(p->ti + 2 * p->dt, p->tf + p->dt, p->dt);
  t = p->ti + 2 * p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    psod_aux(p, cst, vpot, vabc, u1, u2, v1, v2, work.data());
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      corr(cr, ci);
      cs.put(cr, ci);
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      corr(cr, ci);
      et = energy();
      const double fnr = norm2();
      fnt = fnr * fnr;
      if (absorb)
        *info = 0;
      else if (drifted(et, e0, fnt, f0))
        *info = 1;
      rs.put(t, et, cr, ci, cr * cr + ci * ci, fnt);
    }
  }
  et = energy();
  fnt = norm2();
  if (!absorb && drifted(et, e0, fnt, f0)) *info = 1;  // with ABSORB the test sets 0 (psod.f:197)
  if (absorb) *info = 0;
  if (nrows) *nrows = rs.n;
  return cs.n;
}

// ef.f:20-60  EF
extern "C" double orc_ef(int shape, const double* par, double t) {
  const double FAT = +2.1132e-9;
  const double FATE = +2.29371276e+17 * 3.335664e-28;
  const double FATT = +1.5192676;
  const double PI = +3.14159265358979323846;
  const double e0 = par[0], tp = par[1], omg = par[2], t0 = par[3], sni = par[4];
  if (shape == 1) {
    double ef = e0 * std::exp(-4.0 * 0.693147181 * (t - t0) * (t - t0) / (tp * tp)) *
                std::cos(omg * t * FATT + sni);
    return ef * FATE;
  }
  if (shape == 2) {
    const int kl = (int)par[5];
    const double a1 = 1.0 / (2.0 * kl);
    const double tpa = tp / std::pow((double)0.693147181f, a1);  // REAL literal
    return FAT * std::sqrt(e0 * std::exp(-std::pow((t - t0) / tpa, 2.0 * kl))) *
           std::cos(omg * t * FATT + sni);
  }
  if (shape == 3) {
    double ef = e0 * std::cos(PI * (t - t0) / tp) * std::cos(PI * (t - t0) / tp) *
                std::cos(omg * (t - t0) * FATT + sni);
    return ef * FATE;
  }
  return 0.0;
}

// ppsod.f:64-400  PPSOD's propagation
extern "C" int orc_ppsod(const orc_prop_t* p, const double* vp, const double* vabc,
                         const double* dm, int shape, const double* par, double* u1, double* v1,
                         double* u2, double* v2, double* c_re, double* c_im, int c_cap) {
  const int n = npts(p);
  CSink cs{c_re, c_im, c_cap};
  const double cst = 2.0 * p->dt / ORC_SHFS;
  std::vector<double> u0(u1, u1 + n), v0(v1, v1 + n), work(n), veff(n);
  for (int i = 0; i < n; ++i) {
    u2[i] = u0[i];
    v2[i] = v0[i];
  }
  auto chpot = [&](double t) {  // chpot.f:44-51
    const double e = orc_ef(shape, par, t);
    for (int i = 0; i < n; ++i) veff[i] = vp[i] - dm[i] * e;
  };
  auto corr = [&]() {
    cs.put(orc_fcorrel(n, u0.data(), u2) + orc_fcorrel(n, v0.data(), v2),
           orc_fcorrel(n, u0.data(), v2) - orc_fcorrel(n, v0.data(), u2));
  };
  corr();
  double t = p->ti;
  chpot((t + p->dt) / 2.0);
  psod_aux(p, cst / 4.0, veff.data(), vabc, u1, u2, v1, v2, work.data());
  chpot(t + p->dt);
  psod_aux(p, cst / 2.0, veff.data(), vabc, u1, u2, v1, v2, work.data());
  int mc = 1;
  if (mc == p->lc) {
    mc = 0;
    corr();
  }
  for (int i = 0; i < n; ++i) {  // ppsod.f:373-376
    u1[i] = u0[i];
    v1[i] = v0[i];
  }
  t = p->ti + p->dt;
  const long nf = std::lround((p->tf + p->dt / 2.0 - t) / p->dt);
  for (long k = 1; k <= nf; ++k) {
    t = t + p->dt;
    chpot(t);
    psod_aux(p, cst, veff.data(), vabc, u1, u2, v1, v2, work.data());
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      corr();
    }
  }
  return cs.n;
}

// ---------------------------------------------------------------------------
// Symmetric tridiagonal eigensolver (stands in for DSTEVX('V','A'),
// dstevx.f).  Implicit-shift QL iteration with Wilkinson shifts on a copy of
// (d, e), accumulating the rotations into Z.  Eigenvalues sorted ascending.
// ---------------------------------------------------------------------------
extern "C" int orc_tridiag_eig(int n, const double* d_in, const double* e_in, double* w,
                               double* z) {
  std::vector<double> d(d_in, d_in + n), e(n, 0.0);
  for (int i = 0; i + 1 < n; ++i) e[i] = e_in[i];
  for (int i = 0; i < n * n; ++i) z[i] = 0.0;
  for (int i = 0; i < n; ++i) z[i + n * i] = 1.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-17 * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) return 1;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
      double s = 1.0, c = 1.0, pp = 0.0;
      int i = m - 1;
      bool underflow = false;
      for (; i >= l; --i) {
        double f = s * e[i], bb = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= pp;
          e[m] = 0.0;
          underflow = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - pp;
        r = (d[i] - g) * s + 2.0 * c * bb;
        pp = s * r;
        d[i + 1] = g + pp;
        g = c * r - bb;
        for (int k = 0; k < n; ++k) {  // rotate columns i, i+1 of Z
          double zf = z[k + n * (i + 1)];
          z[k + n * (i + 1)] = s * z[k + n * i] + c * zf;
          z[k + n * i] = c * z[k + n * i] - s * zf;
        }
      }
      if (underflow) continue;
      d[l] -= pp;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  // sort ascending
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (d[ord[j]] < d[ord[i]]) std::swap(ord[i], ord[j]);
  std::vector<double> zz(z, z + n * n);
  for (int i = 0; i < n; ++i) {
    w[i] = d[ord[i]];
    for (int k = 0; k < n; ++k) z[k + n * i] = zz[k + n * ord[i]];
  }
  return 0;
}

// ---------------------------------------------------------------------------
// lnz.f:76-119 (LNZ) with reort.f:65-80 (REORT, classical Gram-Schmidt)
// Builds mp Lanczos vectors of H from start vector s into L (n x mp,
// column-major), alpha al[mp], beta bt[mp].  Returns false when the start
// vector is zero (lnz.f:90 BT0.EQ.0 branch).
// ---------------------------------------------------------------------------
static bool lanczos(int ndim, const int* np, const double* shm, const double* vpot, int n,
                    int mp, const double* s, double* L, double* al, double* bt) {
  std::vector<double> work(s, s + n), vi(n, 0.0), v0(n), rv(mp);
  for (long i = 0; i < (long)n * mp; ++i) L[i] = 0.0;
  double bt0 = orc_ecnorm(n, work.data());
  if (bt0 == 0.0) return false;
  for (int it = 0; it < mp; ++it) {
    for (int j = 0; j < n; ++j) {
      v0[j] = vi[j];
      vi[j] = work[j] / bt0;
      L[j + (long)n * it] = vi[j];
    }
    orc_au(ndim, np, shm, vpot, vi.data(), work.data());
    double sum1 = 0.0;
    for (int j = 0; j < n; ++j) {
      work[j] = work[j] - bt0 * v0[j];
      sum1 = sum1 + vi[j] * work[j];
    }
    al[it] = sum1;
    for (int j = 0; j < n; ++j) work[j] = work[j] - al[it] * vi[j];
    const int m = it + 1;  // REORT against the it+1 stored vectors
    for (int q = 0; q < m; ++q) {
      double r = 0.0;
      for (int j = 0; j < n; ++j) r = r + work[j] * L[j + (long)n * q];
      rv[q] = r;
    }
    for (int q = 0; q < m; ++q)
      for (int j = 0; j < n; ++j) work[j] = work[j] - rv[q] * L[j + (long)n * q];
    bt[it] = orc_ecnorm(n, work.data());
    bt0 = bt[it];
  }
  return true;
}

// sil.f:70-181 PLNZAUX: one short-iterative-Lanczos step, real and imaginary
// parts propagated by separate Krylov bases.
static int sil_step(const orc_prop_t* p, int mp, const double* vpot, const double* vabc,
                    double cst, double* u, double* v) {
  const int n = npts(p);
  std::vector<double> L((size_t)n * mp), al(mp), bt(mp), w(mp), q((size_t)mp * mp);
  std::vector<double> a(mp), c(mp), sn(mp), tmp(mp);
  std::vector<double> ur(n, 0.0), ui(n, 0.0), vr(n, 0.0), vi(n, 0.0);
  auto project = [&](const double* x, double* y) {  // y = Q^T L^T x
    for (int k = 0; k < mp; ++k) tmp[k] = orc_fcorrel(n, L.data() + (size_t)n * k, x);
    for (int i = 0; i < mp; ++i) {
      double s = 0.0;
      for (int j = 0; j < mp; ++j) s = s + q[j + mp * i] * tmp[j];
      y[i] = s;
    }
  };
  auto expand = [&](const double* y, double* x) {  // x = L Q y
    for (int j = 0; j < mp; ++j) {
      double s = 0.0;
      for (int i = 0; i < mp; ++i) s = s + q[j + mp * i] * y[i];
      tmp[j] = s;
    }
    for (int k = 0; k < n; ++k) {
      double s = 0.0;
      for (int j = 0; j < mp; ++j) s = s + L[k + (size_t)n * j] * tmp[j];
      x[k] = s;
    }
  };
  // real part: e^{-iH dt} u = cos(H dt) u - i sin(H dt) u
  if (lanczos(p->ndim, p->np, p->shm, vpot, n, mp, u, L.data(), al.data(), bt.data())) {
    if (orc_tridiag_eig(mp, al.data(), bt.data(), w.data(), q.data())) return -1;
    project(u, a.data());
    for (int i = 0; i < mp; ++i) {
      double e = w[i] * cst;
      double cu = std::cos(e) * a[i];
      sn[i] = -std::sin(e) * ((p->quirks & ORC_Q_SIL_INPLACE) ? cu : a[i]);
      c[i] = cu;
    }
    expand(c.data(), ur.data());
    expand(sn.data(), ui.data());
  }
  // imaginary part: e^{-iH dt} (i v) = sin(H dt) v + i cos(H dt) v
  if (lanczos(p->ndim, p->np, p->shm, vpot, n, mp, v, L.data(), al.data(), bt.data())) {
    if (orc_tridiag_eig(mp, al.data(), bt.data(), w.data(), q.data())) return -1;
    project(v, a.data());
    for (int i = 0; i < mp; ++i) {
      double e = w[i] * cst;
      sn[i] = std::sin(e) * a[i];
      c[i] = std::cos(e) * a[i];
    }
    expand(c.data(), vi.data());
    expand(sn.data(), vr.data());
  }
  if (p->absorb == ORC_ABS_SMOOTHW) {  // sil.f:171-175
    for (int k = 0; k < n; ++k) {
      u[k] = vabc[k] * (ur[k] + vr[k]);
      v[k] = vabc[k] * (ui[k] + vi[k]);
    }
  } else {
    for (int k = 0; k < n; ++k) {
      u[k] = ur[k] + vr[k];
      v[k] = ui[k] + vi[k];
    }
  }
  return 0;
}

// plnz.f:71-151  PLNZ
extern "C" int orc_plnz(const orc_prop_t* p, const double* vpot, const double* vabc,
                        double* u, double* v, double* c_re, double* c_im, int c_cap,
                        double* rows, int row_cap, int* nrows, int* info) {
  const int n = npts(p);
  RowSink rs{rows, row_cap};
  CSink cs{c_re, c_im, c_cap};
  *info = 0;
  const double cst = p->dt / ORC_SHFS;
  int mp = p->mp;
  if (p->change && mp > p->lmtreort) mp = p->lmtreort;  // lnz.f:64-72 (MP aliased)
  if (p->absorb == ORC_ABS_VOPTIC) return -1;           // real-symmetric Lanczos only
  std::vector<double> u0(u, u + n), v0(v, v + n);
  auto corr = [&](double& cr, double& ci) {
    cr = orc_fcorrel(n, u0.data(), u) + orc_fcorrel(n, v0.data(), v);
    ci = orc_fcorrel(n, u0.data(), v) - orc_fcorrel(n, v0.data(), u);
  };
  auto energy = [&]() {
    return orc_eigenerg(p->ndim, p->np, p->shm, vpot, u) +
           orc_eigenerg(p->ndim, p->np, p->shm, vpot, v);
  };
  double cr, ci;
  corr(cr, ci);
  double ct = cr * cr + ci * ci;  // plnz.f:86 prints |C|^2
  cs.put(cr, ci);
  double et = energy();
  const double e0 = et;
  double fnt = orc_fcorrel(n, u, u) + orc_fcorrel(n, v, v);
  const double f0 = fnt;
  if (p->prtcrl != ORC_PRT_NONE) rs.put(p->ti, et, cr, ci, ct, fnt);
  int mc = 0;
  const int nit = orc_do_count(p->ti + p->dt, p->tf + p->dt, p->dt);
  double t = p->ti + p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    if (sil_step(p, mp, vpot, vabc, cst, u, v)) return -1;  // sil.f:119-120 STOP
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      corr(cr, ci);
      cs.put(cr, ci);
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      corr(cr, ci);
      ct = cr * cr + ci * ci;
      et = energy();
      fnt = orc_fcorrel(n, u, u) + orc_fcorrel(n, v, v);
      if (std::fabs((et - e0) / e0) * 100.0 > p->tol ||
          std::fabs((fnt - f0) / f0) * 100.0 > p->tol)
        *info = 1;
      rs.put(t, et, cr, ci, ct, fnt);
    }
  }
  et = energy();
  fnt = orc_fcorrel(n, u, u) + orc_fcorrel(n, v, v);
  if (std::fabs((et - e0) / e0) * 100.0 > p->tol || std::fabs((fnt - f0) / f0) * 100.0 > p->tol)
    *info = 1;
  if (nrows) *nrows = rs.n;
  return cs.n;
}

// ppsod.f:64-400 with its table: rows of 7 + npr values (T, ET, E0, CR, CI,
// |C|^2, |P_1|^2 .. |P_npr|^2, FNT) as FORMAT 1021 prints them -- ET with the potential of the
// last CHPOT, E0 with VP, P_k = <W_k|psi> (W real, ppsod.f:158-189), FNT the
// norm; C(t) stored in LNZVC as ppsod.f does: C(0) and the start-up sample
// only inside the print test (ppsod.f:145-150, 263-297), the loop's every LC
// steps; INFO = 1 when the norm drifts (no absorber, ppsod.f:434-438)
extern "C" int orc_ppsod_table(const orc_prop_t* p, const double* vp, const double* vabc,
                               const double* dm, int shape, const double* par, int npr,
                               const double* w, double* u1, double* v1, double* u2, double* v2,
                               double* c_re, double* c_im, int c_cap, double* rows, int row_cap,
                               int* nrows, int* info) {
  const int n = npts(p);
  CSink cs{c_re, c_im, c_cap};
  const int ncol = 7 + npr;
  int nr = 0;
  *info = 0;
  const double cst = 2.0 * p->dt / ORC_SHFS;
  std::vector<double> u0(u1, u1 + n), v0(v1, v1 + n), work(n), veff(vp, vp + n);
  for (int i = 0; i < n; ++i) {
    u2[i] = u0[i];
    v2[i] = v0[i];
  }
  auto chpot = [&](double t) {
    const double e = orc_ef(shape, par, t);
    for (int i = 0; i < n; ++i) veff[i] = vp[i] - dm[i] * e;
  };
  double f0 = 0.0;
  auto row = [&](double t) {
    const double cr = orc_fcorrel(n, u0.data(), u2) + orc_fcorrel(n, v0.data(), v2);
    const double ci = orc_fcorrel(n, u0.data(), v2) - orc_fcorrel(n, v0.data(), u2);
    if (rows && nr < row_cap) {
      double* r = rows + (size_t)ncol * nr;
      r[0] = t;
      r[1] = orc_eigenerg(p->ndim, p->np, p->shm, veff.data(), u2) +
             orc_eigenerg(p->ndim, p->np, p->shm, veff.data(), v2);
      r[2] = orc_eigenerg(p->ndim, p->np, p->shm, vp, u2) +
             orc_eigenerg(p->ndim, p->np, p->shm, vp, v2);
      r[3] = cr;
      r[4] = ci;
      r[5] = cr * cr + ci * ci;
      for (int k = 0; k < npr; ++k) {
        const double pr = orc_fcorrel(n, w + (size_t)n * k, u2);
        const double pi = orc_fcorrel(n, w + (size_t)n * k, v2);
        r[6 + k] = pr * pr + pi * pi;
      }
    }
    const double fnt = orc_fcorrel(n, u2, u2) + orc_fcorrel(n, v2, v2);
    if (rows && nr < row_cap) rows[(size_t)ncol * nr + ncol - 1] = fnt;
    ++nr;
    return fnt;
  };
  auto store = [&]() {
    cs.put(orc_fcorrel(n, u0.data(), u2) + orc_fcorrel(n, v0.data(), v2),
           orc_fcorrel(n, u0.data(), v2) - orc_fcorrel(n, v0.data(), u2));
  };
  const bool prt = p->prtcrl != ORC_PRT_NONE;
  if (prt) {
    store();
    f0 = row(p->ti);
  } else {
    cs.put(0.0, 0.0);  // LNZVC(1, .) is not written: a placeholder keeps the rows aligned
    cs.n = 1;
  }
  double t = p->ti;
  chpot((t + p->dt) / 2.0);
  psod_aux(p, cst / 4.0, veff.data(), vabc, u1, u2, v1, v2, work.data());
  chpot(t + p->dt);
  psod_aux(p, cst / 2.0, veff.data(), vabc, u1, u2, v1, v2, work.data());
  int mc = 1;
  t = p->ti + p->dt;
  if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == p->lc)) {
    if (mc == p->lc) {
      mc = 0;
      store();
    }
    row(t);
  }
  for (int i = 0; i < n; ++i) {
    u1[i] = u0[i];
    v1[i] = v0[i];
  }
  t = p->ti + p->dt;
  const long nf = std::lround((p->tf + p->dt / 2.0 - t) / p->dt);
  for (long k = 1; k <= nf; ++k) {
    t = t + p->dt;
    chpot(t);
    psod_aux(p, cst, veff.data(), vabc, u1, u2, v1, v2, work.data());
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      store();
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      const double fnt = row(t);
      if (p->absorb == ORC_ABS_NONE && std::fabs((fnt - f0) / f0) * 100.0 > p->tol) *info = 1;
    }
  }
  if (nrows) *nrows = nr;
  return cs.n;
}

// pplnz.f:139-141  PPLNZ's propagation: DO T = TI+DT, TF+DT/2, DT with the
// potential VP - DM EF(T) (chpot.f) in each PLNZAUX step; C(t) every LC steps
extern "C" int orc_pplnz(const orc_prop_t* p, const double* vp, const double* vabc,
                         const double* dm, int shape, const double* par, double* u, double* v,
                         double* c_re, double* c_im, int c_cap) {
  const int n = npts(p);
  CSink cs{c_re, c_im, c_cap};
  const double cst = p->dt / ORC_SHFS;
  int mp = p->mp;
  if (p->change && mp > p->lmtreort) mp = p->lmtreort;
  if (p->absorb == ORC_ABS_VOPTIC) return -1;
  std::vector<double> u0(u, u + n), v0(v, v + n), veff(n);
  auto corr = [&]() {
    cs.put(orc_fcorrel(n, u0.data(), u) + orc_fcorrel(n, v0.data(), v),
           orc_fcorrel(n, u0.data(), v) - orc_fcorrel(n, v0.data(), u));
  };
  corr();
  int mc = 0;
  const int nit = orc_do_count(p->ti + p->dt, p->tf + p->dt / 2.0, p->dt);
  double t = p->ti + p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    const double e = orc_ef(shape, par, t);
    for (int i = 0; i < n; ++i) veff[i] = vp[i] - dm[i] * e;
    if (sil_step(p, mp, veff.data(), vabc, cst, u, v)) return -1;
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      corr();
    }
  }
  return cs.n;
}

// pplnz.f:76-320 PPLNZ with its table: rows of 6 + npr values (T, ET, E0, CR,
// CI, CT(1..NPR), FNT) as FORMAT 1021 prints them -- CT(1) = |C|^2 and CT(k+1)
// = |<W_k|psi>|^2 for k < NPR (pplnz.f:110-142: the last W read is not
// printed), ET with the potential of the last CHPOT, E0 with VP, FNT the norm
// except on the first row, where it is the norm squared (pplnz.f:146-147);
// C(t) in LNZVC: C(0) inside the print test only, then every LC steps;
// INFO = 1 when a printed row's FNT drifts from the first row's (no absorber,
// pplnz.f:270-274); w: the npr - 1 printed projection vectors
extern "C" int orc_pplnz_table(const orc_prop_t* p, const double* vp, const double* vabc,
                               const double* dm, int shape, const double* par, int npr,
                               const double* w, double* u, double* v, double* c_re,
                               double* c_im, int c_cap, double* rows, int row_cap, int* nrows,
                               int* info) {
  const int n = npts(p);
  CSink cs{c_re, c_im, c_cap};
  const int ncol = 6 + (npr > 0 ? npr : 0);
  int nr = 0;
  *info = 0;
  const double cst = p->dt / ORC_SHFS;
  int mp = p->mp;
  if (p->change && mp > p->lmtreort) mp = p->lmtreort;
  if (p->absorb == ORC_ABS_VOPTIC) return -1;
  std::vector<double> u0(u, u + n), v0(v, v + n), veff(vp, vp + n);
  double f0 = 0.0;
  auto row = [&](double t, bool first) {
    const double cr = orc_fcorrel(n, u0.data(), u) + orc_fcorrel(n, v0.data(), v);
    const double ci = orc_fcorrel(n, u0.data(), v) - orc_fcorrel(n, v0.data(), u);
    const double fnr = orc_fcorrel(n, u, u) + orc_fcorrel(n, v, v);
    const double fnt = first ? fnr * fnr : fnr;
    if (rows && nr < row_cap) {
      double* r = rows + (size_t)ncol * nr;
      r[0] = t;
      r[1] = orc_eigenerg(p->ndim, p->np, p->shm, veff.data(), u) +
             orc_eigenerg(p->ndim, p->np, p->shm, veff.data(), v);
      r[2] = orc_eigenerg(p->ndim, p->np, p->shm, vp, u) + orc_eigenerg(p->ndim, p->np, p->shm, vp, v);
      r[3] = cr;
      r[4] = ci;
      if (npr >= 1) r[5] = cr * cr + ci * ci;
      for (int k = 1; k < npr; ++k) {
        const double pr = orc_fcorrel(n, w + (size_t)n * (k - 1), u);
        const double pi = orc_fcorrel(n, w + (size_t)n * (k - 1), v);
        r[5 + k] = pr * pr + pi * pi;
      }
      r[ncol - 1] = fnt;
    }
    ++nr;
    return fnt;
  };
  auto store = [&]() {
    cs.put(orc_fcorrel(n, u0.data(), u) + orc_fcorrel(n, v0.data(), v),
           orc_fcorrel(n, u0.data(), v) - orc_fcorrel(n, v0.data(), u));
  };
  if (p->prtcrl != ORC_PRT_NONE) {
    store();
    f0 = row(p->ti, true);
  } else {
    cs.put(0.0, 0.0);  // LNZVC(1, .) is not written: a placeholder keeps the rows aligned
    cs.n = 1;
  }
  int mc = 0;
  const int nit = orc_do_count(p->ti + p->dt, p->tf + p->dt / 2.0, p->dt);
  double t = p->ti + p->dt;
  for (int it = 0; it < nit; ++it, t = t + p->dt) {
    const double e = orc_ef(shape, par, t);
    for (int i = 0; i < n; ++i) veff[i] = vp[i] - dm[i] * e;
    if (sil_step(p, mp, veff.data(), vabc, cst, u, v)) return -1;
    mc = mc + 1;
    if (mc == p->lc) {
      mc = 0;
      store();
    }
    if (p->prtcrl == ORC_PRT_YES || (p->prtcrl == ORC_PRT_PARTIAL && mc == 0)) {
      const double fnt = row(t, false);
      if (p->absorb == ORC_ABS_NONE && std::fabs((fnt - f0) / f0) * 100.0 > p->tol) *info = 1;
    }
  }
  if (nrows) *nrows = nr;
  return cs.n;
}

// ---------------------------------------------------------------------------
// Spectrum stage
// ---------------------------------------------------------------------------

// espec.f:1545-1576 (one correlation function, ND = 1): mirror C(-t) = C(t)*
// onto 2^MF points; c_re/c_im hold the MC = 2^(MF-1) stored samples.
extern "C" void orc_total_correlation(int mf, const double* c_re, const double* c_im,
                                      double* u, double* v) {
  const int mc = (1 << mf) / 2;
  for (int i = 0; i < 2 * mc; ++i) u[i] = v[i] = 0.0;
  for (int i = 1; i <= mc; ++i) {  // 1-based as in the Fortran
    u[mc + i - 1] = u[mc + i - 1] + c_re[i - 1];
    u[mc - i + 1] = u[mc + i - 1];
    v[mc + i - 1] = v[mc + i - 1] + c_im[i - 1];
    v[mc - i + 1] = -v[mc + i - 1];
  }
  u[0] = u[0] + c_re[mc - 1];
  v[0] = v[0] + c_im[mc - 1];
  v[0] = -v[0];
}

// hwhm.f:59-77  energy shift and exponential lifetime damping
extern "C" void orc_hwhm(int mf, double dtf, double tf, double tal, double de, double* u,
                         double* v) {
  const int n = 1 << mf;
  const double dem = -de * 1.5192676;
  const double ta = tal * 1.5192676;
  for (int i = 0; i < n; ++i) {
    double t = -tf + (double)i * dtf;
    double cs = std::cos(dem * t), sn = std::sin(dem * t);
    double cstl = std::exp(-std::fabs(t) * ta);
    double ui = u[i];
    u[i] = cs * u[i] - sn * v[i];
    v[i] = cs * v[i] + sn * ui;
    u[i] = cstl * u[i];
    v[i] = cstl * v[i];
  }
}

// cfft.f:6-63  FFTNT: in-place radix-2 decimation-in-frequency DFT with
// bit reversal; itype = -1 gives the inverse transform scaled by 1/N.
extern "C" void orc_fftnt(double* x, double* y, int n, int m, int itype, int quirks) {
  if (n == 1) return;
  const double twopi = (quirks & ORC_Q_FFTNT_SP) ? (double)6.283185307179586476925287f
                                                 : 6.283185307179586476925287;
  if (itype == -1)
    for (int i = 0; i < n; ++i) y[i] = -y[i];
  const double pstep = twopi / n;
  int n2 = n;
  for (int k = 0; k < m; ++k) {
    int n1 = n2;
    n2 = n2 / 2;
    int ie = n / n1, ia = 1;
    for (int j = 1; j <= n2; ++j) {
      double a = (ia - 1) * pstep;
      double c = std::cos(a), s = std::sin(a);
      ia = ia + ie;
      for (int i = j; i <= n; i += n1) {
        int l = i + n2;
        double xt = x[i - 1] - x[l - 1];
        x[i - 1] = x[i - 1] + x[l - 1];
        double yt = y[i - 1] - y[l - 1];
        y[i - 1] = y[i - 1] + y[l - 1];
        x[l - 1] = c * xt + s * yt;
        y[l - 1] = c * yt - s * xt;
      }
    }
  }
  int j = 1;
  for (int i = 1; i <= n - 1; ++i) {
    if (i < j) {
      std::swap(x[j - 1], x[i - 1]);
      std::swap(y[j - 1], y[i - 1]);
    }
    int k = n / 2;
    while (k < j) {
      j = j - k;
      k = k / 2;
    }
    j = j + k;
  }
  if (itype == -1)
    for (int i = 0; i < n; ++i) {
      y[i] = -y[i] / n;
      x[i] = x[i] / n;
    }
}

// spectrumtd.f:58-109  window (.SG or none), half swap, inverse FFTNT.
// en[i] receives the energy printed beside natural index i (without DE).
extern "C" int orc_spectrumtd(int window_sg, int mf, double dtf, double tf, double wp,
                              double de, double* u, double* v, double* en, int quirks) {
  const int n = 1 << mf;
  double enc = 1.0 / (n * dtf) * 1.519829846003e-1;
  enc = enc * ORC_FATE;
  double e = -n / 2.0 * enc;
  (void)de;
  if (window_sg) {
    const double tmax = n * dtf;
    const double taux = tmax * tmax / (std::log(1.0 / wp) * std::log(1.0 / wp));
    for (int i = 0; i < n; ++i) {
      double t = -tf + (double)i * dtf;
      double cstl = std::exp(-t * t / taux);
      u[i] = cstl * u[i];
      v[i] = cstl * v[i];
    }
  }
  for (int i = 0; i < n / 2; ++i) {
    std::swap(u[i], u[n / 2 + i]);
    std::swap(v[i], v[n / 2 + i]);
  }
  orc_fftnt(u, v, n, mf, -1, quirks);
  for (int i = n / 2; i < n; ++i) {
    en[i] = e;
    e = e + enc;
  }
  for (int i = 0; i < n / 2; ++i) {
    en[i] = e;
    e = e + enc;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Batched 1D split-operator scan (CPU baseline): independent packets, each
// propagated with the reference step (spofft.f:120-191) and C(t) of every
// step (pspofft.f:115-123, LC = 1).  Packets are spread over nthreads host
// threads through a shared packet counter.
// ---------------------------------------------------------------------------
// The same step as orc_spo_step for a 1D packet without absorber, with the
// cosines and sines of the V half-phase and of the kinetic phase computed
// once per packet instead of every step (spofft.f recomputes them, 3N DCOS
// and DSIN per step).  Every product and sum is the one orc_spo_step forms,
// in the same order, so the results are bit for bit the same; only the
// repeated sincos calls are gone, which makes this CPU baseline faster per
// core than the reference's own loop.
struct SpoCached {
  int n = 0;
  std::vector<double> cv, sv;  // cos/sin(cst2 V(i))
  std::vector<double> ck, sk;  // cos/sin(cst1 TC(i))
};

static void spo_cached_init(SpoCached& c, int n, double cst1, double cst2, const double* tc,
                            const double* vpot) {
  c.n = n;
  c.cv.resize(n);
  c.sv.resize(n);
  c.ck.resize(n);
  c.sk.resize(n);
  for (int i = 0; i < n; ++i) {
    sincos(cst2 * vpot[i], &c.sv[i], &c.cv[i]);
    sincos(cst1 * tc[i], &c.sk[i], &c.ck[i]);
  }
}

static void spo_step_cached(const SpoCached& c, double b, int quirks, double* u, double* v) {
  const int n = c.n, nh = n / 2;
  const double *cv = c.cv.data(), *sv = c.sv.data();
  for (int i = 0; i < nh; ++i) {
    const double c1 = cv[i], s1 = sv[i];
    double ua = c1 * u[i] + s1 * v[i];
    double va = c1 * v[i] - s1 * u[i];
    const double c2 = cv[i + nh], s2 = sv[i + nh];
    u[i] = c2 * u[i + nh] + s2 * v[i + nh];
    v[i] = c2 * v[i + nh] - s2 * u[i + nh];
    u[i + nh] = ua;
    v[i + nh] = va;
  }
  int np[3] = {n, 1, 1};
  fft_all_axes(1, np, n, u, v, 1);
  for (int i = 0; i < n; ++i) {
    const double cc = c.ck[i], s = c.sk[i];
    double un = cc * u[i] + s * v[i];
    if (quirks & ORC_Q_SPO_INPLACE) {
      u[i] = un;
      v[i] = cc * v[i] - s * u[i];
    } else {
      v[i] = cc * v[i] - s * u[i];
      u[i] = un;
    }
  }
  fft_all_axes(1, np, n, u, v, -1);
  for (int i = 0; i < nh; ++i) {
    const double c1 = cv[i + nh], s1 = sv[i + nh];
    double ua = c1 * b * u[i] + s1 * b * v[i];
    double va = c1 * b * v[i] - s1 * b * u[i];
    const double c2 = cv[i], s2 = sv[i];
    double un = c2 * b * u[i + nh] + s2 * b * v[i + nh];
    double vn = c2 * b * v[i + nh] - s2 * b * u[i + nh];
    u[i] = un;
    v[i] = vn;
    u[i + nh] = ua;
    v[i + nh] = va;
  }
}

extern "C" int orc_spo_batch(int npk, const int* off, const double* sh, const double* sm,
                             const double* vpot, double* u, double* v, double dt_fs,
                             int nsteps, int quirks, double* c_re, double* c_im,
                             int nthreads) {
  std::atomic<int> next{0};
  auto worker = [&]() {
    SpoCached cache;
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= npk) return;
      const int n = off[k + 1] - off[k];
      double* uk = u + off[k];
      double* vk = v + off[k];
      const double* vp = vpot + off[k];
      std::vector<double> u0(uk, uk + n), v0(vk, vk + n), tc(n);
      double b;
      int np[3] = {n, 1, 1};
      orc_digt(1, np, sh + k, sm + k, tc.data(), &b, 0);
      const double cst1 = dt_fs / ORC_SHFS, cst2 = dt_fs / (2.0 * ORC_SHFS);
      spo_cached_init(cache, n, cst1, cst2, tc.data(), vp);
      double* cr = c_re + (size_t)k * (nsteps + 1);
      double* ci = c_im + (size_t)k * (nsteps + 1);
      for (int s = 0; s <= nsteps; ++s) {
        if (s > 0) spo_step_cached(cache, b, quirks, uk, vk);
        cr[s] = orc_fcorrel(n, u0.data(), uk) + orc_fcorrel(n, v0.data(), vk);
        ci[s] = orc_fcorrel(n, u0.data(), vk) - orc_fcorrel(n, v0.data(), uk);
      }
    }
  };
  if (nthreads < 1) nthreads = 1;
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  return 0;
}

// ---------------------------------------------------------------------------
// Initial-state eigensolver (LANCZSG, lanczsc.f:56-120)
// ---------------------------------------------------------------------------

// rans.f:38-39  NSEED = MOD(NSEED*L + NC, M), RAN = NSEED/M
extern "C" double orc_ran(int* nseed) {
  const long long L = 1029, NC = 221591, M = 1048576;
  *nseed = (int)(((long long)*nseed * L + NC) % M);
  return (double)*nseed / (double)M;
}

// lanczsc.f:56-62: NSEED = 1, N draws discarded, then N draws per state
extern "C" void orc_lcg_start(int n, int nstates, double* out) {
  int seed = 1;
  for (int i = 0; i < n; ++i) orc_ran(&seed);
  for (int k = 0; k < nstates; ++k)
    for (int i = 0; i < n; ++i) out[(long)k * n + i] = orc_ran(&seed);
}

// LNZ (lnz.f:76-119) whose REORT set (reort.f:65-80) also holds nlock
// locked eigenvectors: all dot products of the step first, then all updates.
static void lanczos_locked(int ndim, const int* np, const double* shm, const double* vpot, int n,
                           int mp, const double* s, const double* lock, int nlock, double* L,
                           double* al, double* bt) {
  std::vector<double> work(s, s + n), vi(n, 0.0), v0(n), rv(mp + nlock);
  for (long i = 0; i < (long)n * mp; ++i) L[i] = 0.0;
  double bt0 = orc_ecnorm(n, work.data());
  for (int it = 0; it < mp; ++it) {
    for (int j = 0; j < n; ++j) {
      v0[j] = vi[j];
      vi[j] = work[j] / bt0;
      L[j + (long)n * it] = vi[j];
    }
    orc_au(ndim, np, shm, vpot, vi.data(), work.data());
    double sum1 = 0.0;
    for (int j = 0; j < n; ++j) {
      work[j] = work[j] - bt0 * v0[j];
      sum1 = sum1 + vi[j] * work[j];
    }
    al[it] = sum1;
    for (int j = 0; j < n; ++j) work[j] = work[j] - al[it] * vi[j];
    for (int q = 0; q < nlock; ++q) {
      double r = 0.0;
      for (int j = 0; j < n; ++j) r = r + work[j] * lock[j + (long)n * q];
      rv[q] = r;
    }
    for (int q = 0; q <= it; ++q) {
      double r = 0.0;
      for (int j = 0; j < n; ++j) r = r + work[j] * L[j + (long)n * q];
      rv[nlock + q] = r;
    }
    for (int q = 0; q < nlock; ++q)
      for (int j = 0; j < n; ++j) work[j] = work[j] - rv[q] * lock[j + (long)n * q];
    for (int q = 0; q <= it; ++q)
      for (int j = 0; j < n; ++j) work[j] = work[j] - rv[nlock + q] * L[j + (long)n * q];
    bt[it] = orc_ecnorm(n, work.data());
    bt0 = bt[it];
  }
}

// For each state K: the start vector made orthogonal to the states already
// found, LNZ (m steps) with those states locked in the REORT set, the lowest
// Ritz pair of the tridiagonal matrix (DSTEVX('V','I',...) in the reference;
// QL here), v = L y normalised by ECNORM (lanczsc.f:99-113), and -- in place
// of the reference's sum |VI(I) - VIAUX(I)| test, whose index is the loop
// bound (lanczsc.f:103) -- the true residual |H v - theta v| against tol.
// (Without locking, the reference's K-th Ritz vector can settle on a higher
// state; espec.f:896-903 restricts LANCZSG to the ground state.)  matvecs
// counts H*v.  Returns 0, or 1 when a state needed more than maxrest restarts.
extern "C" int orc_eig_lanczsg(int ndim, const int* np, const double* shm, const double* vpot,
                               int nstates, int m, double tol, int maxrest, const double* start,
                               double* evals, double* evecs, double* resid, int* matvecs) {
  int n = 1;
  for (int a = 0; a < ndim; ++a) n *= np[a];
  std::vector<double> L((size_t)n * m), al(m), bt(m), w(m), z((size_t)m * m), v(n), hv(n);
  int rc = 0;
  for (int K = 0; K < nstates; ++K) {
    for (int i = 0; i < n; ++i) v[i] = start[(long)K * n + i];
    int count = 0;
    double res = 0.0, theta = 0.0;
    bool done = false;
    for (int rs = 0; rs < maxrest && !done; ++rs) {
      for (int q = 0; q < K; ++q) {  // project out the locked states
        const double* e = evecs + (long)q * n;
        const double c = orc_fcorrel(n, e, v.data());
        for (int i = 0; i < n; ++i) v[i] = v[i] - c * e[i];
      }
      lanczos_locked(ndim, np, shm, vpot, n, m, v.data(), evecs, K, L.data(), al.data(),
                     bt.data());
      count += m;
      orc_tridiag_eig(m, al.data(), bt.data(), w.data(), z.data());
      theta = w[0];
      for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < m; ++j) s += z[j] * L[i + (size_t)n * j];
        v[i] = s;
      }
      const double fatn = orc_ecnorm(n, v.data());
      for (int i = 0; i < n; ++i) v[i] = v[i] / fatn;
      orc_au(ndim, np, shm, vpot, v.data(), hv.data());
      count += 1;
      double r2 = 0.0;
      for (int i = 0; i < n; ++i) {
        const double r = hv[i] - theta * v[i];
        r2 += r * r;
      }
      res = std::sqrt(r2);
      done = res <= tol;
    }
    if (!done) rc = 1;
    evals[K] = theta;
    resid[K] = res;
    matvecs[K] = count;
    for (int i = 0; i < n; ++i) evecs[(long)K * n + i] = v[i];
  }
  return rc;
}

// ---------------------------------------------------------------------------
// potfuncs.f:3-497  POT1D / POT2D / POT3D: the analytic potentials, chosen by
// the first prefix test of POTCH that matches, in the reference's order.
// ---------------------------------------------------------------------------
static bool pot_is(const char* potch, const char* p) {
  return std::strncmp(potch, p, std::strlen(p)) == 0;
}

extern "C" double orc_pot1d(const char* potch, const double* cst, double rx) {
  const double* c = cst - 1;  // CST(1..) as in the Fortran
  if (pot_is(potch, ".OHS")) return 5.0e-1 * c[2] * std::pow(rx - c[1], 2);  // :63-64
  if (pot_is(potch, ".DOHS"))                                                 // :66-68
    return 5.0e-1 * c[2] * std::pow(rx - c[1], 2) +
           c[5] * std::exp(std::pow(rx - c[3], 2) / std::pow(c[4], 2));
  if (pot_is(potch, ".MORSEM"))  // :70-79
    return c[3] * (std::exp(-2.0 * c[2] * (rx - c[1])) - 2.0 * std::exp(-c[2] * (rx - c[1])));
  if (pot_is(potch, ".ANTI-MORSEM"))  // :85-92
    return c[3] / 2.0 * (std::exp(-2.0 * c[2] * (rx - c[1])) + 2.0 * std::exp(-c[2] * (rx - c[1])));
  if (pot_is(potch, ".MOD-MORSE"))  // :100-102
    return c[3] * std::pow(c[4] - std::exp(-c[2] * (rx - c[1])), 2) + c[5];
  if (pot_is(potch, ".MORSE")) return c[3] * std::pow(1.0 - std::exp(-c[2] * (rx - c[1])), 2);
  if (pot_is(potch, ".ANTI-MORSE"))
    return c[3] / 2.0 * std::pow(1.0 + std::exp(-c[2] * (rx - c[1])), 2);
  if (pot_is(potch, ".DMORSE"))  // :113-115
    return c[3] * std::pow(1.0 - std::exp(-c[4] * (rx - c[1])), 2) +
           c[5] * std::exp(-c[6] * std::pow(rx - c[2], 2));
  if (pot_is(potch, ".STEP")) return (rx >= c[1] && rx <= c[2]) ? 0.0 : c[3];
  if (pot_is(potch, ".BARRIER")) return (rx >= c[1] && rx <= c[2]) ? c[3] : 0.0;
  if (pot_is(potch, ".CONST") || pot_is(potch, ".FREE")) return c[1];
  return std::nan("");  // the reference prints an error and STOPs
}

extern "C" double orc_pot3d(const char* potch, const double* cst, double rx, double ry,
                            double rz) {
  const double* c = cst - 1;
  if (pot_is(potch, ".OHS"))
    return 5.0e-1 * c[2] * std::pow(rx - c[1], 2) + 5.0e-1 * c[4] * std::pow(ry - c[3], 2) +
           5.0e-1 * c[6] * std::pow(rz - c[5], 2);
  if (pot_is(potch, ".STEP"))
    return (rx >= c[1] && rx <= c[2] && ry >= c[3] && ry <= c[4] && rz >= c[5] && rz <= c[6])
               ? 0.0 : c[7];
  if (pot_is(potch, ".BARRIER"))  // :425-431, the third test on RY as written
    return (rx >= c[1] && rx <= c[2] && ry >= c[3] && ry <= c[4] && ry >= c[5] && ry <= c[6])
               ? c[7] : 0.0;
  if (pot_is(potch, ".LEPS")) {  // :433-487
    const double a = c[10], b = c[11], g = c[12];
    const double q1 = 5.0e-1 * (orc_pot1d(".MORSEM", cst, rx) +
                                (1 - a) / (1 + a) * orc_pot1d(".ANTI-MORSEM", cst, rx));
    const double q2 = 5.0e-1 * (orc_pot1d(".MORSEM", cst + 3, ry) +
                                (1 - b) / (1 + b) * orc_pot1d(".ANTI-MORSEM", cst + 3, ry));
    const double q3 = 5.0e-1 * (orc_pot1d(".MORSEM", cst + 6, rz) +
                                (1 - g) / (1 + g) * orc_pot1d(".ANTI-MORSEM", cst + 6, rz));
    const double j1 = 5.0e-1 * (orc_pot1d(".MORSEM", cst, rx) -
                                (1 - a) / (1 + a) * orc_pot1d(".ANTI-MORSEM", cst, rx));
    const double j2 = 5.0e-1 * (orc_pot1d(".MORSEM", cst + 3, ry) -
                                (1 - b) / (1 + b) * orc_pot1d(".ANTI-MORSEM", cst + 3, ry));
    const double j3 = 5.0e-1 * (orc_pot1d(".MORSEM", cst + 6, rz) -
                                (1 - g) / (1 + g) * orc_pot1d(".ANTI-MORSEM", cst + 6, rz));
    return q1 + q2 + q3 -
           std::sqrt(j1 * j1 + j2 * j2 + j3 * j3 - j1 * j2 - j2 * j3 - j1 * j3);
  }
  if (pot_is(potch, ".CONST") || pot_is(potch, ".FREE")) return c[1];
  return std::nan("");
}

extern "C" double orc_pot2d(const char* potch, const double* sm, const double* cst, double rx,
                            double ry) {
  const double* c = cst - 1;
  const double* m = sm - 1;
  if (pot_is(potch, ".OHS"))
    return 5.0e-1 * c[2] * std::pow(rx - c[1], 2) + 5.0e-1 * c[4] * std::pow(ry - c[3], 2);
  if (pot_is(potch, ".MORSE"))
    return c[3] * std::pow(1.0 - std::exp(-c[2] * (rx - c[1])), 2) +
           c[6] * std::pow(1.0 - std::exp(-c[5] * (ry - c[4])), 2);
  if (pot_is(potch, ".LSM") || pot_is(potch, ".LS")) {  // :214-233
    const double v1a = c[3] * (1.0 - std::exp(-c[2] * std::pow(rx - c[1], 2) / (2.0 * rx + 1.0e-99)));
    const double v1b =
        c[5] * (1.0 - std::exp(-c[4] * std::pow(ry - rx - c[1], 2) / (2.0 * (ry - c[1]) + 1.0e-99)));
    if (!pot_is(potch, ".LSM")) return v1a + v1b;
    const double v2 = c[2] * std::pow(1.0 - std::exp(-c[7] * (ry - c[6])), 2);
    return v1a + v1b + v2;
  }
  if (pot_is(potch, ".LBH_CC") || pot_is(potch, ".LBH")) {  // :234-253
    double rxa = rx, rya = ry;
    if (pot_is(potch, ".LBH_CC")) {
      rya = ry / std::sqrt(m[2] * m[3] * (m[1] + m[2] + m[3]) / (std::pow(m[2] + m[3], 2) * m[1]));
      rxa = rx + m[2] * rya / (m[2] + m[3]) - rya;
    }
    const double vab = c[1] * std::exp(-1.0 / c[2] * rxa);
    const double vbc = c[3] * (std::exp(-2.0 * c[4] * (rya - c[5])) - 2.0 * std::exp(-c[4] * (rya - c[5])));
    return vab + vbc;
  }
  if (pot_is(potch, ".LEPS_CC")) {
    const double rya =
        ry / std::sqrt(m[2] * m[3] * (m[1] + m[2] + m[3]) / (std::pow(m[2] + m[3], 2) * m[1]));
    const double rxa = rx - m[2] * rya / (m[2] + m[3]);
    const double rza = std::sqrt(rxa * rxa + rya * rya - 2.0 * rxa * rya * std::cos(c[13]));
    return orc_pot3d(".LEPS", cst, rxa, rya, rza);
  }
  if (pot_is(potch, ".LEPS")) {
    const double rz = std::sqrt(rx * rx + ry * ry - 2.0 * rx * ry * std::cos(c[13]));
    return orc_pot3d(".LEPS", cst, rx, ry, rz);
  }
  if (pot_is(potch, ".WELLXY"))
    return ((rx >= c[1] && rx <= c[2]) ? 0.0 : c[3]) + ((ry >= c[4] && ry <= c[5]) ? 0.0 : c[6]);
  if (pot_is(potch, ".WELLX")) return (rx >= c[1] && rx <= c[2]) ? 0.0 : c[3];
  if (pot_is(potch, ".WELLY")) return (ry >= c[1] && ry <= c[2]) ? 0.0 : c[3];
  if (pot_is(potch, ".WELL"))
    return (rx >= c[1] && rx <= c[2] && ry >= c[3] && ry <= c[4]) ? 0.0 : c[5];
  if (pot_is(potch, ".BARRIERXY"))
    return ((rx >= c[1] && rx <= c[2]) ? c[3] : 0.0) + ((ry >= c[4] && ry <= c[5]) ? c[6] : 0.0);
  if (pot_is(potch, ".BARRIERX")) return (rx >= c[1] && rx <= c[2]) ? c[3] : 0.0;
  if (pot_is(potch, ".BARRIERY")) return (ry >= c[1] && ry <= c[2]) ? c[3] : 0.0;
  if (pot_is(potch, ".BARRIER"))
    return (rx >= c[1] && rx <= c[2] && ry >= c[3] && ry <= c[4]) ? c[5] : 0.0;
  if (pot_is(potch, ".CONST") || pot_is(potch, ".FREE")) return c[1];
  return std::nan("");
}

// gvpot.f:1-111  GVPOT: the potential on the grid (x fastest) and, with
// SHIFTP, the shift by its minimum (1D and 3D: when above 1e-6; 2D: when its
// magnitude is); 1D returns XMIN.  The 3D loop takes RX from the K index
// (gvpot.f:96) when quirk3d is set.
extern "C" void orc_gvpot(int shiftp, const char* potch, int ndim, const int* np,
                          const double* xi, const double* sm, const double* sh,
                          const double* cst, int quirk3d, double* vpot, double* xmin) {
  double aux = 1.0e+99;
  if (ndim == 1) {
    for (int i = 0; i < np[0]; ++i) {
      const double rx = xi[0] + i * sh[0];
      vpot[i] = orc_pot1d(potch, cst, rx);
      if (shiftp && vpot[i] < aux) {
        aux = vpot[i];
        *xmin = rx;
      }
    }
    if (shiftp && aux > 1.0e-6)
      for (int i = 0; i < np[0]; ++i) vpot[i] -= aux;
  } else if (ndim == 2) {
    for (int j = 0; j < np[1]; ++j) {
      const double ry = xi[1] + j * sh[1];
      for (int i = 0; i < np[0]; ++i) {
        const double rx = xi[0] + i * sh[0];
        const long l = i + (long)j * np[0];
        vpot[l] = orc_pot2d(potch, sm, cst, rx, ry);
        if (shiftp && vpot[l] < aux) aux = vpot[l];
      }
    }
    if (shiftp && std::fabs(aux) > 1.0e-6)
      for (long l = 0; l < (long)np[0] * np[1]; ++l) vpot[l] -= aux;
  } else {
    for (int k = 0; k < np[2]; ++k) {
      const double rz = xi[2] + k * sh[2];
      for (int j = 0; j < np[1]; ++j) {
        const double ry = xi[1] + j * sh[1];
        for (int i = 0; i < np[0]; ++i) {
          const double rx = xi[0] + (quirk3d ? k : i) * sh[0];
          const long l = i + (long)j * np[0] + (long)k * np[0] * np[1];
          vpot[l] = orc_pot3d(potch, cst, rx, ry, rz);
          if (shiftp && vpot[l] < aux) aux = vpot[l];
        }
      }
    }
    if (shiftp && aux > 1.0e-6)
      for (long l = 0; l < (long)np[0] * np[1] * np[2]; ++l) vpot[l] -= aux;
  }
}
