// spond.cu -- split-operator propagation (PSPOFFT / PSPOFFTAUX, pspofft.f,
// spofft.f:64-200) on one 2D or 3D grid, FP64 or mixed (FP32 data, FP64
// tables), and the plan behind espec_spond_* (include/espec_gpu.h).
//
// Line transforms: one warp per line of N = 32 P points (P = 1..16); lane l
// holds points 32 j + l in register j.  Forward = four-step: a P-point DFT
// in registers (radix-2 decimation in frequency), twiddles W_N^(l k1), then a
// 32-point DFT across the lanes by __shfl_xor butterflies (decimation in
// frequency): lane l, register r ends with frequency brev_P(r) + P brev_32(l).
// The inverse is the exact mirror with conjugate twiddles (unnormalised).
// Between the passes of a step each row stays in that permuted frequency
// order; only the kinetic pass needs the frequencies, via its table.
//
// Passes per step (the V half-steps of consecutive steps merged, g = h^2):
//   2D: x pass [inverse x, C(t), x-space phase, forward x]; y pass [forward y,
//       kinetic phase, inverse y]
//   3D: x pass; y pass [forward y]; z pass [forward z, kinetic, inverse z];
//       y pass [inverse y]
// Strided passes stage a tile of 8 adjacent x columns in shared memory.  The
// fftshift swaps of spofft.f:120-133/178-191 cancel and are not done; the
// 1/N of the reference's B factor is folded into the kinetic table.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>
#include <vector>

#include "cplx.cuh"
#include "espec_gpu.h"
#include "espec_internal.h"
#include "cplx_io.cuh"

namespace espec {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxWarps = 8;  // lines per CTA (one warp each); fewer on small grids

template <typename R>
__device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
__device__ __forceinline__ cpx<R> cmulc(cpx<R> a, cpx<R> b) {  // a * conj(b)
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename R>
__device__ __forceinline__ cpx<R> shx(cpx<R> v, int m) {
  return mk(__shfl_xor_sync(kFull, v.x, m), __shfl_xor_sync(kFull, v.y, m));
}
__host__ __device__ __forceinline__ int brev_bits(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}
template <int P>
constexpr int log2i() {
  return P <= 1 ? 0 : 1 + log2i<P / 2>();
}
// Fixed rotations: FP64 as (cos, sin) applied by a complex product; FP32 as
// three lifting shears (RotF), whose rounding is unbiased -- a rounded
// (cos, sin) pair has |w| != 1 and a fixed-angle product loses or gains norm
// systematically, step after step.
template <typename R>
struct Rot;
template <>
struct Rot<double> {
  using type = RotD;
  static __device__ __forceinline__ RotD make(double k_over_n) {  // exp(-2 pi i k/n)
    RotD r;
    sincospi(-2.0 * k_over_n, &r.s, &r.c);
    return r;
  }
};
template <>
struct Rot<float> {
  using type = RotF;
  static __device__ __forceinline__ RotF make(double k_over_n) {
    return make_rotf(-6.283185307179586476925287 * k_over_n);
  }
};
template <typename R>
__device__ __forceinline__ typename Rot<R>::type twid(int k, int n) {
  return Rot<R>::make((double)k / (double)n);
}

// x-space and kinetic factors: FP64 complex, or FP32 lifting rotation with a
// magnitude (the sign of a removed pi folded into it)
struct PhF {
  float t, s, ag;
};
template <typename R>
struct Ph;
template <>
struct Ph<double> {
  using type = cpx<double>;
};
template <>
struct Ph<float> {
  using type = PhF;
};
__host__ __device__ __forceinline__ cpx<double> apply_ph(cpx<double> p, cpx<double> v) {
  return mk(v.x * p.x - v.y * p.y, v.x * p.y + v.y * p.x);
}
__host__ __device__ __forceinline__ cpx<float> apply_ph(PhF p, cpx<float> v) {
  float x = v.x * p.ag, y = v.y * p.ag;
  x = fmaf(-p.t, y, x);
  y = fmaf(p.s, x, y);
  x = fmaf(-p.t, y, x);
  return mk(x, y);
}
// e^{i phi} times a, as stored factors
__host__ __device__ inline PhF make_phf(double phi, double a) {
  const RotF r = make_rotf(phi);
  PhF o;
  o.t = r.t;
  o.s = r.s;
  o.ag = (float)(r.g * a);
  return o;
}

template <typename R, int P>
struct WarpFft {
  static constexpr int LP = log2i<P>();
  using T = typename Rot<R>::type;
  T wl[5];                         // lane stages m = 16 .. 1: W_2m^(lane & (m-1))
  T wb[P];                         // W_N^(lane k1(r))
  T wr[P > 1 ? P / 2 : 1];         // W_P^q, q < P/2
  int lane;

  // every twiddle is W_N^k, k < N: read from the line's table (built once
  // per plan in FP64, tw_table_kernel)
  __device__ void init(const T* tab) {
    constexpr int N = 32 * P;
    lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const int m = 16 >> s;
      wl[s] = tab[(lane & (m - 1)) * (N / (2 * m))];
    }
#pragma unroll
    for (int r = 0; r < P; ++r) wb[r] = tab[lane * brev_bits(r, LP)];
#pragma unroll
    for (int q = 0; q < (P > 1 ? P / 2 : 1); ++q) wr[q] = tab[q * 32];
  }
  __device__ void forward(cpx<R>* v) const {
#pragma unroll
    for (int h = P / 2; h >= 1; h /= 2)
#pragma unroll
      for (int b = 0; b < P; b += 2 * h)
#pragma unroll
        for (int q = 0; q < h; ++q) {
          const cpx<R> a = v[b + q], c = v[b + q + h];
          v[b + q] = a + c;
          v[b + q + h] = rot<false>(wr[q * (P / (2 * h))], a - c);
        }
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = rot<false>(wb[r], v[r]);
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const int m = 16 >> s;
      const bool up = lane & m;
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const cpx<R> mine = v[r], other = shx(mine, m);
        v[r] = up ? rot<false>(wl[s], other - mine) : mine + other;
      }
    }
  }
  __device__ void inverse(cpx<R>* v) const {
#pragma unroll
    for (int s = 4; s >= 0; --s) {
      const int m = 16 >> s;
      const bool up = lane & m;
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const cpx<R> mine = up ? rot<true>(wl[s], v[r]) : v[r];
        const cpx<R> other = shx(mine, m);
        v[r] = up ? other - mine : mine + other;
      }
    }
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = rot<true>(wb[r], v[r]);
#pragma unroll
    for (int h = 1; h <= P / 2; h *= 2)
#pragma unroll
      for (int b = 0; b < P; b += 2 * h)
#pragma unroll
        for (int q = 0; q < h; ++q) {
          const cpx<R> a = v[b + q], t = rot<true>(wr[q * (P / (2 * h))], v[b + q + h]);
          v[b + q] = a + t;
          v[b + q + h] = a - t;
        }
  }
};

template <typename R>
struct NdArgs {
  int nx, ny, nz, ndim;
  cpx<R>* psi;            // state
  const double2* psi0;    // psi(0), natural order (FIRST pass input)
  const double2* psi_start;  // resume / diagnostics: natural-order state read instead
  double2* psi_out;       // psi(TF), natural order (LAST pass output)
  using PhT = typename Ph<R>::type;
  const PhT* g;           // x-space factors, natural order
  const PhT* h;
  const PhT* hm;
  const double2* w;       // conj(psi0) hm, for C(t) (FP64 in both forms)
  const PhT* K;           // kinetic factors in the kinetic pass's layout
  const double* kq_c;     // reference-defect form: cos / sin(CST1 TC) in that layout
  const double* kq_s;
  double kq_scale;
  double2* cpart;         // C(t) partial sums [step][x-pass CTA]
  const typename Rot<R>::type* tw[3];  // W_n^k tables of the x, y, z line lengths
  int step;
  // second-order differences (psodfft.f / sodfft.f:64-126): dst <- dst - i f
  // (vc src + T src) [+ f ab src, or times the mask], natural order
  const double2* sod_src;
  double2* sod_dst;
  const double* vc;   // CST V
  const double* ab;   // CST VABC (.VOPTIC) or the .SMOOTHW mask
  double f;
  int kabs;           // 0 none, 1 complex potential, 2 mask
};

// W_n^k = exp(-2 pi i k / n), k < n, in the form the line transforms apply
template <typename R>
__global__ void tw_table_kernel(typename Rot<R>::type* tab, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) tab[k] = twid<R>(k, n);
}

enum { kFirst = 0, kMid = 1, kLast = 2, kFwd0 = 3, kSodUpd = 4 };

// x pass: one warp per row, 8 rows per CTA
template <typename R, int P, int MODE>
__global__ void __launch_bounds__(256) x_pass(NdArgs<R> a) {
  constexpr int N = 32 * P;
  __shared__ double2 s_c[kMaxWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const long row = (long)blockIdx.x * nw + warp;
  const long nrows = (long)a.ny * a.nz;
  WarpFft<R, P> fft;
  fft.init(a.tw[0]);
  cpx<R> v[P];
  double cr = 0.0, ci = 0.0;
  if (row < nrows) {
    const long base = row * N;
    if (MODE == kFirst) {
      const double2* src = a.psi_start ? a.psi_start : a.psi0;
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const long x = base + 32 * j + lane;
        const double2 p = src[x];
        cr += p.x * p.x + p.y * p.y;  // C(0) = <psi0|psi0> (not used when resuming)
        v[j] = apply_ph(a.h[x], mk((R)p.x, (R)p.y));
      }
    } else if (MODE == kSodUpd) {
      // T src by the inverse of the transformed copy, then the leapfrog update
#pragma unroll
      for (int j = 0; j < P; ++j) v[j] = a.psi[base + 32 * j + lane];
      fft.inverse(v);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const long x = base + 32 * j + lane;
        const double2 sj = a.sod_src[x], dj = a.sod_dst[x];
        const double vc = a.vc[x];
        const double hx = fma(vc, sj.x, (double)v[j].x), hy = fma(vc, sj.y, (double)v[j].y);
        double ox = fma(a.f, hy, dj.x), oy = fma(-a.f, hx, dj.y);
        if (a.kabs == 1) {
          const double abf = a.f * a.ab[x];
          ox = fma(abf, sj.x, ox);
          oy = fma(abf, sj.y, oy);
        } else if (a.kabs == 2) {
          ox *= a.ab[x];
          oy *= a.ab[x];
        }
        a.sod_dst[x] = make_double2(ox, oy);
        const double2 wj = a.w[x];  // conj(psi0)
        cr += wj.x * ox - wj.y * oy;
        ci += wj.x * oy + wj.y * ox;
      }
    } else if (MODE == kFwd0) {  // plain forward transform of a natural-order state
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const double2 p = a.psi_start[base + 32 * j + lane];
        v[j] = mk((R)p.x, (R)p.y);
      }
    } else {
#pragma unroll
      for (int j = 0; j < P; ++j) v[j] = a.psi[base + 32 * j + lane];
      fft.inverse(v);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const long x = base + 32 * j + lane;
        const double2 wj = a.w[x];
        cr += wj.x * (double)v[j].x - wj.y * (double)v[j].y;
        ci += wj.x * (double)v[j].y + wj.y * (double)v[j].x;
        v[j] = apply_ph(MODE == kLast ? a.hm[x] : a.g[x], v[j]);
      }
    }
    if (MODE == kSodUpd) {
      // written above
    } else if (MODE == kLast) {
#pragma unroll
      for (int j = 0; j < P; ++j)
        a.psi_out[base + 32 * j + lane] = make_double2((double)v[j].x, (double)v[j].y);
    } else {
      fft.forward(v);
#pragma unroll
      for (int j = 0; j < P; ++j) a.psi[base + 32 * j + lane] = v[j];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cr += __shfl_xor_sync(kFull, cr, o);
    ci += __shfl_xor_sync(kFull, ci, o);
  }
  if (lane == 0) s_c[warp] = make_double2(cr, ci);
  __syncthreads();
  if (threadIdx.x == 0 && a.cpart) {
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < nw; ++i) {
      sr += s_c[i].x;
      si += s_c[i].y;
    }
    a.cpart[(long)a.step * gridDim.x + blockIdx.x] = make_double2(sr, si);
  }
}

// C(0) = sum |psi0|^2 as x-pass-shaped partials (nb blocks)
__global__ void c0_kernel(const double2* psi0, long n, double2* part) {
  __shared__ double red[256];
  const long lo = n * blockIdx.x / gridDim.x, hi = n * (blockIdx.x + 1) / gridDim.x;
  double s = 0.0;
  for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) s += psi0[i].x * psi0[i].x + psi0[i].y * psi0[i].y;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(red[0], 0.0);
}

// SOD tables: vc = CST V, ab = CST VABC or the mask, w = conj(psi0)
__global__ void sod_setup_nd_kernel(long n, const double* vpot, const double* vabc, int kabs,
                                    double cst, const double2* psi0, double* vc, double* ab,
                                    double2* w) {
  const long x = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  vc[x] = cst * vpot[x];
  ab[x] = kabs == 1 ? cst * vabc[x] : (kabs == 2 ? vabc[x] : 0.0);
  w[x] = make_double2(psi0[x].x, -psi0[x].y);
}

// EFFT4 (eigenergfft.f:58-100) and the norm of a natural-order state psi
// given its forward transform khat in the passes' storage order:
// sum V |psi|^2 + (1/N) sum TC |khat|^2 and sum |psi|^2, per-CTA partials
__global__ void nd_energy_kernel(const double2* psi, const double* vpot, const cpx<double>* khat,
                                 const double* tcp, long n, double rn, double2* part) {
  __shared__ double2 red[256];
  double e = 0.0, nr = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const double2 p = psi[i];
    const double a2 = p.x * p.x + p.y * p.y;
    const cpx<double> k = khat[i];
    e += vpot[i] * a2 + rn * tcp[i] * (k.x * k.x + k.y * k.y);
    nr += a2;
  }
  red[threadIdx.x] = make_double2(e, nr);
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[threadIdx.x].x += red[threadIdx.x + o].x;
      red[threadIdx.x].y += red[threadIdx.x + o].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

enum { kFwd = 0, kInv = 1, kKin = 2 };

// strided pass along axis 1 (y) or 2 (z): CTA = blockDim/32 adjacent x columns
// of one line set, staged through shared memory; warp w transforms column w
template <typename R, int P, int MODE, bool QUIRK>
__global__ void __launch_bounds__(256) axis_pass(NdArgs<R> a, int axis) {
  constexpr int N = 32 * P;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int kTile = blockDim.x >> 5;  // adjacent x columns per CTA, one warp each
  cpx<R>* tile = reinterpret_cast<cpx<R>*>(sm_raw);  // [N][kTile + 1]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ntx = a.nx / kTile;
  const long xt = blockIdx.x % ntx, other = blockIdx.x / ntx;
  long stride, base;
  if (axis == 1) {  // lines along y: x = 8 xt + c, z = other
    stride = a.nx;
    base = other * (long)a.nx * a.ny + xt * kTile;
  } else {          // lines along z: x = 8 xt + c, y = other
    stride = (long)a.nx * a.ny;
    base = other * (long)a.nx + xt * kTile;
  }
  for (int e = threadIdx.x; e < N * kTile; e += blockDim.x) {
    const int t = e / kTile, c = e % kTile;
    tile[t * (kTile + 1) + c] = a.psi[base + t * stride + c];
  }
  __syncthreads();
  WarpFft<R, P> fft;
  fft.init(a.tw[axis]);
  cpx<R> v[P];
#pragma unroll
  for (int j = 0; j < P; ++j) v[j] = tile[(32 * j + lane) * (kTile + 1) + warp];
  if (MODE == kFwd || MODE == kKin) fft.forward(v);
  if (MODE == kKin) {
    // kinetic table line: x position and the other coordinate
    const long line = (xt * kTile + warp) + (long)a.nx * other;
    const long kb = line * N;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const long f = kb + 32 * j + lane;
      if constexpr (QUIRK) {
        // spofft.f:148-154 as written: V(I) uses the already updated U(I)
        const double c = a.kq_c[f], s = a.kq_s[f];
        const double un = c * (double)v[j].x + s * (double)v[j].y;
        const double vn = c * (double)v[j].y - s * un;
        v[j] = mk((R)(un * a.kq_scale), (R)(vn * a.kq_scale));
      } else {
        v[j] = apply_ph(a.K[f], v[j]);
      }
    }
  }
  if (MODE == kInv || MODE == kKin) fft.inverse(v);
#pragma unroll
  for (int j = 0; j < P; ++j) tile[(32 * j + lane) * (kTile + 1) + warp] = v[j];
  __syncthreads();
  for (int e = threadIdx.x; e < N * kTile; e += blockDim.x) {
    const int t = e / kTile, c = e % kTile;
    a.psi[base + t * stride + c] = tile[t * (kTile + 1) + c];
  }
}

// C(t) of each step: the x-pass partial sums in CTA order
__global__ void csum_kernel(const double2* cpart, int nparts, int nsteps, int first,
                            double2* c_out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x + first;
  if (s > nsteps) return;
  double sr = 0.0, si = 0.0;
  for (int i = 0; i < nparts; ++i) {
    const double2 p = cpart[(long)s * nparts + i];
    sr += p.x;
    si += p.y;
  }
  c_out[s] = make_double2(sr, si);
}

// x-space tables (spofft.f:120-133, 162-191): h = e^{-i cst2 V} (x e^{cst2
// VABC} for .VOPTIC), g = h^2 (x mask), hm = h mask, w = conj(psi0) hm
__device__ __forceinline__ void put_ph(cpx<double>* o, double phi, double a) {
  double s, c;
  sincos(phi, &s, &c);
  *o = mk(c * a, s * a);
}
__device__ __forceinline__ void put_ph(PhF* o, double phi, double a) { *o = make_phf(phi, a); }

template <typename R>
__global__ void nd_setup_kernel(long n, const double* vpot, const double* vabc, int absorb,
                                double cst2, const double2* psi0, typename Ph<R>::type* g,
                                typename Ph<R>::type* h, typename Ph<R>::type* hm, double2* w) {
  const long x = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  const double th = cst2 * vpot[x];
  double hmag = 1.0, mask = 1.0;
  if (absorb == ESPEC_ABS_VOPTIC) hmag = exp(cst2 * vabc[x]);
  if (absorb == ESPEC_ABS_SMOOTHW) mask = vabc[x];
  double s1, c1, s2, c2;
  sincos(th, &s1, &c1);
  sincos(2.0 * th, &s2, &c2);
  (void)s2;
  (void)c2;
  put_ph(g + x, -2.0 * th, hmag * hmag * mask);
  put_ph(h + x, -th, hmag);
  put_ph(hm + x, -th, hmag * mask);
  const double hr = c1 * hmag * mask, hi = -s1 * hmag * mask;
  const double2 p = psi0[x];
  w[x] = make_double2(p.x * hr + p.y * hi, p.x * hi - p.y * hr);
}

}  // namespace
}  // namespace espec

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
using namespace espec;

struct espec_spond_plan {
  int ndim = 2, np[3] = {1, 1, 1};
  long n = 0;
  double sh[3] = {1, 1, 1}, sm[3] = {1, 1, 1};
  double dt_fs = 0.0;
  int precision = ESPEC_FP64, absorb = 0, quirks = 0, method = ESPEC_SPO;
  double2* d_prev = nullptr;  // SOD: psi(t - dt), natural order
  double* d_sod = nullptr;    // SOD: vc, ab (n each)
  bool loaded = false;
  void* d_psi = nullptr;      // cpx<R> state
  double2* d_psi0 = nullptr;
  double2* d_out = nullptr;
  double* d_vpot = nullptr;
  double* d_vabc = nullptr;
  void* d_tab = nullptr;      // g, h, hm, w, K (cpx<R>)
  double* d_kq = nullptr;     // quirk cos/sin tables
  double2* d_cpart = nullptr;
  double2* d_c = nullptr;
  void* d_tw[3] = {nullptr, nullptr, nullptr};
  int c_cap = -1, xblocks = 0;
  bool has_state = false;          // d_out holds the state of the last run
  // energy diagnostics (FP64 in both forms)
  cpx<double>* d_khat = nullptr;
  double* d_tcp = nullptr;         // TC in the passes' storage order
  RotD* d_tw64[3] = {nullptr, nullptr, nullptr};
  double2* d_epart = nullptr;
  HostStage stage;                 // host transfers: (re | im) blocks, contiguous
};

namespace {

bool line_ok(int n) { return n == 32 || n == 64 || n == 128 || n == 256 || n == 512; }

// frequency held at stored position pos of a line of n = 32 P points
int freq_of(int pos, int n) {
  const int P = n / 32, lp = P == 1 ? 0 : (P == 2 ? 1 : (P == 4 ? 2 : (P == 8 ? 3 : 4)));
  return brev_bits(pos / 32, lp) + P * brev_bits(pos % 32, 5);
}

const double kDigtTwoPi = 6.283185307;  // dkeft.f:38

void digt_axis_host(int n, double sh, double sm, double* t) { espec::digt_1d(n, sh, sm, t); }

// kinetic table TC in the reference's FFT order (x fastest): the outer sum of
// the axis tables, or with ESPEC_Q_DIGT_ND the 2D/3D loops of dkeft.f:80-137
// as they are written (only TC(1..NP1) is filled)
void digt_nd(const espec_spond_plan* p, std::vector<double>& tc) {
  const int nx = p->np[0], ny = p->np[1], nz = p->ndim > 2 ? p->np[2] : 1;
  tc.assign((size_t)p->n, 0.0);
  if (p->quirks & ESPEC_Q_DIGT_ND) {
    double dp[3];
    for (int a = 0; a < p->ndim; ++a) dp[a] = kDigtTwoPi / (p->np[a] * p->sh[a]);
    if (p->ndim == 2) {
      double p1 = 0, p2 = 0;
      for (int j = 0; j < ny / 2; ++j) {
        for (int i = 0; i < nx / 2; ++i) {
          tc[i] = p1 * p1 / (2 * p->sm[0]) + p2 * p2 / (2 * p->sm[1]);
          p1 = p1 + dp[0];
        }
        p2 = p2 + dp[1];
      }
      p1 = -(p1 + dp[0]);
      p2 = -(p2 + dp[1]);
      for (int j = ny / 2; j < ny; ++j) {
        for (int i = nx / 2; i < nx; ++i) {
          tc[i] = p1 * p1 / (2 * p->sm[0]) + p2 * p2 / (2 * p->sm[1]);
          p1 = p1 + dp[0];
        }
        p2 = p2 + dp[1];
      }
    } else {
      double p1 = 0, p2 = 0, p3 = 0;
      for (int k = 0; k < nz / 2; ++k) {
        for (int j = 0; j < ny / 2; ++j) {
          for (int i = 0; i < nx / 2; ++i) {
            tc[i] = p1 * p1 / (2 * p->sm[0]) + p2 * p2 / (2 * p->sm[1]) +
                    p3 * p3 / (2 * p->sm[2]);
            p1 = p1 + dp[0];
          }
          p2 = p2 + dp[1];
        }
        p3 = p3 + dp[2];
      }
      p1 = -(p1 + dp[0]);
      p2 = -(p2 + dp[1]);
      p3 = -(p3 + dp[2]);
      for (int k = nz / 2; k < nz; ++k) {
        for (int j = ny / 2; j < ny; ++j) {
          for (int i = nx / 2; i < nx; ++i) {
            tc[i] = p1 * p1 / (2 * p->sm[0]) + p2 * p2 / (2 * p->sm[1]) +
                    p3 * p3 / (2 * p->sm[2]);
            p1 = p1 + dp[0];
          }
          p2 = p2 + dp[1];
        }
        p3 = p3 + dp[2];
      }
    }
    return;
  }
  std::vector<double> t[3];
  for (int a = 0; a < p->ndim; ++a) {
    t[a].resize(p->np[a]);
    digt_axis_host(p->np[a], p->sh[a], p->sm[a], t[a].data());
  }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        tc[i + (size_t)nx * (j + (size_t)ny * k)] =
            t[0][i] + t[1][j] + (p->ndim > 2 ? t[2][k] : 0.0);
}

#define ND_CK(call)                                          \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_); \
  } while (0)

// table block: g, h, hm (PhT) | w (double2) | K (PhT), n entries each
template <typename R>
struct NdTabs {
  using PhT = typename Ph<R>::type;
  PhT *g, *h, *hm, *K;
  double2* w;
  static size_t bytes(long n) { return (size_t)n * (4 * sizeof(PhT) + sizeof(double2)); }
  NdTabs(void* base, long n) {
    char* b = (char*)base;
    w = (double2*)b;
    g = (PhT*)(b + 16 * (size_t)n);
    h = g + n;
    hm = h + n;
    K = hm + n;
  }
};

inline cpx<double> k_factor(double th, long n, double) {
  return mk(std::cos(th) / n, -std::sin(th) / n);
}
inline PhF k_factor(double th, long n, float) { return make_phf(-th, 1.0 / n); }
inline cpx<double> k_real(double v, double) { return mk(v, 0.0); }
inline PhF k_real(double v, float) { return make_phf(0.0, v); }

inline int sod_kabs(const espec_spond_plan* p) {
  if (p->absorb == ESPEC_ABS_VOPTIC) return 1;
  if (p->absorb == ESPEC_ABS_SMOOTHW && !(p->quirks & ESPEC_Q_SOD_SMOOTHW)) return 2;
  return 0;  // sodfft.f:108 compares 7 characters with '.SMOOTHW': never true
}

template <typename R>
int build_tables(espec_spond_plan* p, cudaStream_t st) {
  const long n = p->n;
  NdTabs<R> tb(p->d_tab, n);
  const double cst1 = p->dt_fs / ESPEC_SHFS, cst2 = p->dt_fs / (2.0 * ESPEC_SHFS);
  const bool sod = p->method == ESPEC_SOD;
  const double cst_sod = 2.0 * p->dt_fs / ESPEC_SHFS;  // psodfft.f:81
  if (sod) {
    sod_setup_nd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        n, p->d_vpot, p->d_vabc, sod_kabs(p), cst_sod, p->d_psi0, p->d_sod, p->d_sod + n, tb.w);
  } else {
    nd_setup_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        n, p->d_vpot, p->d_vabc, p->absorb, cst2, p->d_psi0, tb.g, tb.h, tb.hm, tb.w);
  }
  ND_CK(cudaGetLastError());
  // kinetic factors in the kinetic pass's layout: line (x position, other
  // position), position along the kinetic axis; frequencies mirrored to the
  // reference's FFT sign (fft3d.f: ISN = +1 is exp(+2 pi i jk/n))
  std::vector<double> tc;
  digt_nd(p, tc);
  const int nx = p->np[0], ny = p->np[1], nz = p->ndim > 2 ? p->np[2] : 1;
  const int ka = p->ndim - 1;  // kinetic axis: y (2D) or z (3D)
  const int nk = p->np[ka];
  std::vector<typename Ph<R>::type> K((size_t)n);
  std::vector<double> qc, qs;
  const bool quirk = (p->quirks & ESPEC_Q_SPO_INPLACE) != 0;
  if (quirk) {
    qc.resize((size_t)n);
    qs.resize((size_t)n);
  }
  const long nlines = n / nk;
  for (long line = 0; line < nlines; ++line) {
    const int px = (int)(line % nx);
    const int po = (int)(line / nx);  // y position (3D) or unused (2D)
    const int fx = (nx - freq_of(px, nx)) % nx;
    const int fy2 = p->ndim > 2 ? (ny - freq_of(po, ny)) % ny : 0;
    for (int pos = 0; pos < nk; ++pos) {
      const int fk = (nk - freq_of(pos, nk)) % nk;
      size_t idx;
      if (p->ndim == 2) idx = fx + (size_t)nx * fk;
      else idx = fx + (size_t)nx * (fy2 + (size_t)ny * fk);
      const double th = cst1 * tc[idx];
      const size_t o = (size_t)line * nk + pos;
      if (sod) {
        K[o] = k_real(cst_sod * tc[idx] / n, R(0));  // CST TC B (sodfft.f:100-104,119)
      } else {
        K[o] = k_factor(th, n, R(0));
      }
      if (quirk) {
        qc[o] = std::cos(th);
        qs[o] = std::sin(th);
      }
    }
  }
  (void)nz;
  ND_CK(cudaMemcpyAsync(tb.K, K.data(), sizeof(K[0]) * n, cudaMemcpyHostToDevice, st));
  if (quirk) {
    ND_CK(cudaMemcpyAsync(p->d_kq, qc.data(), 8 * n, cudaMemcpyHostToDevice, st));
    ND_CK(cudaMemcpyAsync(p->d_kq + n, qs.data(), 8 * n, cudaMemcpyHostToDevice, st));
  }
  ND_CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
  return ESPEC_OK;
}

// warps per CTA: 8, or fewer when that leaves SMs idle (2 CTAs per SM wanted)
int warps_for(long lines) {
  int w = kMaxWarps;
  while (w > 1 && lines / w < 2 * 148) w /= 2;
  return w;
}

template <typename R, int P>
cudaError_t launch_x(int mode, const NdArgs<R>& a, int blocks, cudaStream_t st) {
  const long rows = (long)a.ny * a.nz;
  const int w = warps_for(rows);
  blocks = (int)((rows + w - 1) / w);
  switch (mode) {
    case kFirst: x_pass<R, P, kFirst><<<blocks, 32 * w, 0, st>>>(a); break;
    case kMid: x_pass<R, P, kMid><<<blocks, 32 * w, 0, st>>>(a); break;
    case kFwd0: x_pass<R, P, kFwd0><<<blocks, 32 * w, 0, st>>>(a); break;
    case kSodUpd:
      if constexpr (sizeof(R) == 8) {
        x_pass<R, P, kSodUpd><<<blocks, 32 * w, 0, st>>>(a);
        break;
      }
      return cudaErrorInvalidValue;  // SOD plans are FP64
    case kLast: x_pass<R, P, kLast><<<blocks, 32 * w, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_x_n(int nx, int mode, const NdArgs<R>& a, int blocks, cudaStream_t st) {
  switch (nx) {
    case 32: return launch_x<R, 1>(mode, a, blocks, st);
    case 64: return launch_x<R, 2>(mode, a, blocks, st);
    case 128: return launch_x<R, 4>(mode, a, blocks, st);
    case 256: return launch_x<R, 8>(mode, a, blocks, st);
    default: return launch_x<R, 16>(mode, a, blocks, st);
  }
}

template <typename R, int P, int MODE, bool Q>
cudaError_t launch_axis1(const NdArgs<R>& a, int axis, long, cudaStream_t st) {
  static DeviceFlags attr;
  {
    const size_t smax = sizeof(cpx<R>) * 32 * P * (kMaxWarps + 1);
    cudaError_t e = set_max_smem_once(attr, axis_pass<R, P, MODE, Q>, smax);
    if (e != cudaSuccess) return e;
  }
  const long other = axis == 1 ? a.nz : a.ny;  // line sets beside the x tiles
  const int w = warps_for((long)a.nx * other);
  const long blocks = (long)(a.nx / w) * other;
  const size_t smem = sizeof(cpx<R>) * 32 * P * (w + 1);
  axis_pass<R, P, MODE, Q><<<(unsigned)blocks, 32 * w, smem, st>>>(a, axis);
  return cudaGetLastError();
}

template <typename R, int P>
cudaError_t launch_axis_p(int mode, bool quirk, const NdArgs<R>& a, int axis, long blocks,
                          cudaStream_t st) {
  if (mode == kFwd) return launch_axis1<R, P, kFwd, false>(a, axis, blocks, st);
  if (mode == kInv) return launch_axis1<R, P, kInv, false>(a, axis, blocks, st);
  if constexpr (sizeof(R) == 8) {
    if (quirk) return launch_axis1<R, P, kKin, true>(a, axis, blocks, st);
  }
  return launch_axis1<R, P, kKin, false>(a, axis, blocks, st);
}

template <typename R>
cudaError_t launch_axis(int n, int mode, bool quirk, const NdArgs<R>& a, int axis, long blocks,
                        cudaStream_t st) {
  switch (n) {
    case 32: return launch_axis_p<R, 1>(mode, quirk, a, axis, blocks, st);
    case 64: return launch_axis_p<R, 2>(mode, quirk, a, axis, blocks, st);
    case 128: return launch_axis_p<R, 4>(mode, quirk, a, axis, blocks, st);
    case 256: return launch_axis_p<R, 8>(mode, quirk, a, axis, blocks, st);
    default: return launch_axis_p<R, 16>(mode, quirk, a, axis, blocks, st);
  }
}

template <typename R>
int run_steps(espec_spond_plan* p, int nsteps, bool from_start, cudaStream_t st) {
  NdArgs<R> a{};
  a.nx = p->np[0];
  a.ny = p->np[1];
  a.nz = p->ndim > 2 ? p->np[2] : 1;
  a.ndim = p->ndim;
  a.psi = (cpx<R>*)p->d_psi;
  a.psi0 = p->d_psi0;
  a.psi_out = p->d_out;
  a.psi_start = from_start ? nullptr : p->d_out;
  const long n = p->n;
  NdTabs<R> tb(p->d_tab, n);
  a.g = tb.g;
  a.h = tb.h;
  a.hm = tb.hm;
  a.w = tb.w;
  a.K = tb.K;
  a.kq_c = p->d_kq;
  a.kq_s = p->d_kq ? p->d_kq + n : nullptr;
  a.kq_scale = 1.0 / (double)n;
  a.cpart = p->d_cpart;
  for (int ax = 0; ax < 3; ++ax)
    a.tw[ax] = (const typename Rot<R>::type*)(ax < p->ndim ? p->d_tw[ax] : nullptr);
  const bool quirk = (p->quirks & ESPEC_Q_SPO_INPLACE) != 0;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int xb = p->xblocks;
  const long yb = 0, zb = 0;  // grid sizes are chosen by the launchers
  cudaError_t e = cudaSuccess;
  auto kin_step = [&]() {
    if (p->ndim == 2) {
      e = launch_axis<R>(ny, kKin, quirk, a, 1, yb, st);
    } else {
      e = launch_axis<R>(ny, kFwd, false, a, 1, yb, st);
      if (e == cudaSuccess) e = launch_axis<R>(nz, kKin, quirk, a, 2, zb, st);
      if (e == cudaSuccess) e = launch_axis<R>(ny, kInv, false, a, 1, yb, st);
    }
  };
  if (nsteps == 0) {
    if (from_start) {
      a.step = 0;
      e = launch_x_n<R>(nx, kFirst, a, xb, st);  // C(0); the state is left in k layout
      if (e != cudaSuccess) return set_cuda_error("x pass", e);
      // psi(TF) = psi(0)
      ND_CK(cudaMemcpyAsync(p->d_out, p->d_psi0, 16 * n, cudaMemcpyDeviceToDevice, st));
    }
    return ESPEC_OK;
  }
  for (int s = 0; s <= nsteps; ++s) {
    a.step = s;
    const int mode = s == 0 ? kFirst : (s == nsteps ? kLast : kMid);
    e = launch_x_n<R>(nx, mode, a, xb, st);
    if (e != cudaSuccess) return set_cuda_error("x pass", e);
    if (s < nsteps) {
      kin_step();
      if (e != cudaSuccess) return set_cuda_error("axis pass", e);
    }
  }
  return ESPEC_OK;
}

// second-order differences on the grid (psodfft.f:77-206): start-up of two
// half steps from psi0 (psodfft.f:120-152), then leapfrog steps; the newest
// state ends in d_out, the one before in d_prev
int run_sod(espec_spond_plan* p, int nsteps, bool from_start, cudaStream_t st) {
  NdArgs<double> a{};
  a.nx = p->np[0];
  a.ny = p->np[1];
  a.nz = p->ndim > 2 ? p->np[2] : 1;
  a.ndim = p->ndim;
  a.psi = (cpx<double>*)p->d_psi;  // transform scratch
  const long n = p->n;
  NdTabs<double> tb(p->d_tab, n);
  a.w = tb.w;
  a.K = tb.K;
  a.vc = p->d_sod;
  a.ab = p->d_sod + n;
  a.kabs = sod_kabs(p);
  a.cpart = p->d_cpart;
  for (int ax = 0; ax < 3; ++ax) a.tw[ax] = ax < p->ndim ? (const RotD*)p->d_tw[ax] : nullptr;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  cudaError_t e = cudaSuccess;
  auto op = [&](const double2* src, double2* dst, double f, int step) {
    a.step = step;
    a.psi_start = src;
    e = launch_x_n<double>(nx, kFwd0, a, 0, st);
    if (e != cudaSuccess) return;
    if (p->ndim == 2) {
      e = launch_axis<double>(ny, kKin, false, a, 1, 0, st);
    } else {
      e = launch_axis<double>(ny, kFwd, false, a, 1, 0, st);
      if (e == cudaSuccess) e = launch_axis<double>(nz, kKin, false, a, 2, 0, st);
      if (e == cudaSuccess) e = launch_axis<double>(ny, kInv, false, a, 1, 0, st);
    }
    if (e != cudaSuccess) return;
    a.sod_src = src;
    a.sod_dst = dst;
    a.f = f;
    e = launch_x_n<double>(nx, kSodUpd, a, 0, st);
  };
  double2* cur = p->d_out;
  double2* prev = p->d_prev;
  int s0 = 1;
  if (from_start) {
    ND_CK(cudaMemcpyAsync(cur, p->d_psi0, 16 * n, cudaMemcpyDeviceToDevice, st));
    ND_CK(cudaMemcpyAsync(prev, p->d_psi0, 16 * n, cudaMemcpyDeviceToDevice, st));
    c0_kernel<<<p->xblocks, 256, 0, st>>>(p->d_psi0, n, p->d_cpart);
    ND_CK(cudaGetLastError());
    if (nsteps >= 1) {
      op(cur, prev, 0.5, 1);  // prev = psi0 - i/2 H psi0
      if (e == cudaSuccess) op(prev, cur, 0.5, 1);  // cur = psi0 - i/2 H prev = psi(dt)
      if (e != cudaSuccess) return set_cuda_error("SOD start-up", e);
      ND_CK(cudaMemcpyAsync(prev, p->d_psi0, 16 * n, cudaMemcpyDeviceToDevice, st));
    }
    s0 = 2;
  }
  for (int s = s0; s <= nsteps; ++s) {
    op(cur, prev, 1.0, s);
    if (e != cudaSuccess) return set_cuda_error("SOD step", e);
    std::swap(cur, prev);
  }
  p->d_out = cur;
  p->d_prev = prev;
  return ESPEC_OK;
}

}  // namespace

namespace espec {
// the N-D kinetic table (TC) in the reference's FFT order, for the drop-ins
void digt_nd_table(int ndim, const int* np, const double* sh, const double* sm, int quirks,
                   double* tc) {
  espec_spond_plan q;
  q.ndim = ndim;
  q.n = 1;
  for (int a = 0; a < ndim; ++a) {
    q.np[a] = np[a];
    q.sh[a] = sh[a];
    q.sm[a] = sm[a];
    q.n *= np[a];
  }
  q.quirks = quirks;
  std::vector<double> t;
  digt_nd(&q, t);
  for (long i = 0; i < q.n; ++i) tc[i] = t[i];
}
}  // namespace espec

extern "C" int espec_spond_create_method(espec_spond_plan** out, int method, int ndim,
                                         const int* np, const double* sh, const double* sm,
                                         double dt_fs, int precision, int absorb, int quirks) {
  if (!out || !np || !sh || !sm) return set_error(ESPEC_EINVAL, "null argument");
  if (method != ESPEC_SPO && method != ESPEC_SOD)
    return set_error(ESPEC_EINVAL, "method must be ESPEC_SPO or ESPEC_SOD");
  if (method == ESPEC_SOD && precision != ESPEC_FP64)
    return set_error(ESPEC_EINVAL, "the SOD propagator runs in FP64");
  const int allowed = method == ESPEC_SOD ? (ESPEC_Q_SOD_SMOOTHW | ESPEC_Q_DIGT_ND)
                                          : (ESPEC_Q_SPO_INPLACE | ESPEC_Q_DIGT_ND);
  if (quirks & ~allowed) return set_error(ESPEC_EINVAL, "quirk not applicable to this method");
  if (ndim != 2 && ndim != 3) return set_error(ESPEC_EINVAL, "ndim must be 2 or 3");
  for (int a = 0; a < ndim; ++a)
    if (!line_ok(np[a]))
      return set_error(ESPEC_EINVAL, "axis sizes must be 32, 64, 128, 256 or 512");
  if (precision != ESPEC_FP64 && precision != ESPEC_MIXED)
    return set_error(ESPEC_EINVAL, "precision must be ESPEC_FP64 or ESPEC_MIXED");
  if (absorb < ESPEC_ABS_NONE || absorb > ESPEC_ABS_SMOOTHW)
    return set_error(ESPEC_EINVAL, "unknown absorber type");
  if ((quirks & ESPEC_Q_SPO_INPLACE) && precision != ESPEC_FP64)
    return set_error(ESPEC_EINVAL, "the reference-defect mode exists for FP64 only");
  auto* p = new espec_spond_plan;
  p->method = method;
  p->ndim = ndim;
  p->n = 1;
  for (int a = 0; a < ndim; ++a) {
    p->np[a] = np[a];
    p->sh[a] = sh[a];
    p->sm[a] = sm[a];
    p->n *= np[a];
  }
  p->dt_fs = dt_fs;
  p->precision = precision;
  p->absorb = absorb;
  p->quirks = quirks;
  {
    const long rows = p->n / np[0];
    const int w = warps_for(rows);
    p->xblocks = (int)((rows + w - 1) / w);  // the x pass's grid (C(t) partials per step)
  }
  const size_t n = (size_t)p->n;
  const size_t cb = precision == ESPEC_FP64 ? 16 : 8;
  int rc = 0;
  auto fail = [&](int code) {
    void* b[] = {p->d_psi,   p->d_psi0,  p->d_out,   p->d_vpot,  p->d_vabc, p->d_tab,
                 p->d_kq,    p->d_cpart, p->d_c,     p->d_tw[0], p->d_tw[1], p->d_tw[2],
                 p->d_prev,  p->d_sod};
    for (void* x : b)
      if (x) cudaFree(x);
    delete p;
    return code;
  };
  if ((rc = ck(cudaMalloc(&p->d_psi, cb * n), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_psi0, 16 * n), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_out, 16 * n), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_vpot, 8 * n), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_vabc, 8 * n), "cudaMalloc"))) return fail(rc);
  const size_t tbytes = precision == ESPEC_FP64 ? NdTabs<double>::bytes((long)n)
                                                : NdTabs<float>::bytes((long)n);
  if ((rc = ck(cudaMalloc(&p->d_tab, tbytes), "cudaMalloc"))) return fail(rc);
  if (quirks & ESPEC_Q_SPO_INPLACE)
    if ((rc = ck(cudaMalloc(&p->d_kq, 16 * n), "cudaMalloc"))) return fail(rc);
  if (method == ESPEC_SOD) {
    if ((rc = ck(cudaMalloc(&p->d_prev, 16 * n), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_sod, 16 * n), "cudaMalloc"))) return fail(rc);
  }
  for (int ax = 0; ax < ndim; ++ax)
    if ((rc = ck(cudaMalloc(&p->d_tw[ax], sizeof(RotD) * np[ax]), "cudaMalloc"))) return fail(rc);
  *out = p;
  return ESPEC_OK;
}

extern "C" int espec_spond_create(espec_spond_plan** out, int ndim, const int* np,
                                  const double* sh, const double* sm, double dt_fs,
                                  int precision, int absorb, int quirks) {
  return espec_spond_create_method(out, ESPEC_SPO, ndim, np, sh, sm, dt_fs, precision, absorb,
                                   quirks);
}

extern "C" int espec_spond_previous(espec_spond_plan* p, double* psi_re, double* psi_im,
                                    int where, void* stream) {
  if (!p || p->method != ESPEC_SOD || !p->has_state)
    return set_error(ESPEC_EINVAL, "previous state exists for run SOD plans only");
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = get_complex(p->stage, p->d_prev, psi_re, psi_im, (size_t)p->n, where, st);
  if (rc) return rc;
  if (where == ESPEC_MEM_HOST) ND_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}

extern "C" int espec_spond_load(espec_spond_plan* p, const double* vpot, const double* vabc,
                                const double* psi_re, const double* psi_im, int where,
                                void* stream) {
  if (!p || !vpot || !psi_re) return set_error(ESPEC_EINVAL, "null argument");
  if (p->absorb != ESPEC_ABS_NONE && !vabc) return set_error(ESPEC_EINVAL, "absorber table missing");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)p->n;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  ND_CK(cudaMemcpyAsync(p->d_vpot, vpot, 8 * n, kind, st));
  if (p->absorb != ESPEC_ABS_NONE) ND_CK(cudaMemcpyAsync(p->d_vabc, vabc, 8 * n, kind, st));
  const int rp = put_complex(p->stage, p->d_psi0, psi_re, psi_im, n, where, st);
  if (rp) return rp;
  const int rc = p->precision == ESPEC_FP64 ? build_tables<double>(p, st)
                                            : build_tables<float>(p, st);
  if (rc) return rc;
  p->has_state = false;
  for (int ax = 0; ax < p->ndim; ++ax) {
    const int nl = p->np[ax];
    if (p->precision == ESPEC_FP64)
      tw_table_kernel<double><<<(nl + 255) / 256, 256, 0, st>>>((RotD*)p->d_tw[ax], nl);
    else
      tw_table_kernel<float><<<(nl + 255) / 256, 256, 0, st>>>((RotF*)p->d_tw[ax], nl);
    ND_CK(cudaGetLastError());
  }
  p->loaded = true;
  return ESPEC_OK;
}

extern "C" int espec_spond_run(espec_spond_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_spond_load has not been called");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->c_cap != nsteps) {
    if (p->d_c) cudaFree(p->d_c);
    if (p->d_cpart) cudaFree(p->d_cpart);
    p->d_c = nullptr;
    p->d_cpart = nullptr;
    ND_CK(cudaMalloc(&p->d_c, sizeof(double2) * ((size_t)nsteps + 1)));
    ND_CK(cudaMalloc(&p->d_cpart, sizeof(double2) * ((size_t)nsteps + 1) * p->xblocks));
    p->c_cap = nsteps;
  }
  const int rc = p->method == ESPEC_SOD
                     ? run_sod(p, nsteps, true, st)
                     : (p->precision == ESPEC_FP64 ? run_steps<double>(p, nsteps, true, st)
                                                   : run_steps<float>(p, nsteps, true, st));
  if (rc) return rc;
  csum_kernel<<<(nsteps + 1 + 255) / 256, 256, 0, st>>>(p->d_cpart, p->xblocks, nsteps, 0,
                                                         p->d_c);
  ND_CK(cudaGetLastError());
  p->has_state = true;
  return ESPEC_OK;
}

extern "C" int espec_spond_continue(espec_spond_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->has_state) return set_error(ESPEC_EINVAL, "continue needs a previous run");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->c_cap != nsteps) {
    if (p->d_c) cudaFree(p->d_c);
    if (p->d_cpart) cudaFree(p->d_cpart);
    p->d_c = nullptr;
    p->d_cpart = nullptr;
    ND_CK(cudaMalloc(&p->d_c, sizeof(double2) * ((size_t)nsteps + 1)));
    ND_CK(cudaMalloc(&p->d_cpart, sizeof(double2) * ((size_t)nsteps + 1) * p->xblocks));
    p->c_cap = nsteps;
  }
  if (nsteps == 0) return ESPEC_OK;
  const int rc = p->method == ESPEC_SOD
                     ? run_sod(p, nsteps, false, st)
                     : (p->precision == ESPEC_FP64 ? run_steps<double>(p, nsteps, false, st)
                                                   : run_steps<float>(p, nsteps, false, st));
  if (rc) return rc;
  csum_kernel<<<(nsteps + 255) / 256, 256, 0, st>>>(p->d_cpart, p->xblocks, nsteps, 1, p->d_c);
  ND_CK(cudaGetLastError());
  return ESPEC_OK;
}

// TC of the diagnostic transform's storage order (all axes permuted)
static int nd_energy_tables(espec_spond_plan* p) {
  std::vector<double> tc;
  digt_nd(p, tc);
  const int nx = p->np[0], ny = p->np[1], nz = p->ndim > 2 ? p->np[2] : 1;
  std::vector<double> tcp((size_t)p->n);
  for (int k = 0; k < nz; ++k) {
    const int fz = p->ndim > 2 ? (nz - freq_of(k, nz)) % nz : 0;
    for (int j = 0; j < ny; ++j) {
      const int fy = (ny - freq_of(j, ny)) % ny;
      for (int i = 0; i < nx; ++i) {
        const int fx = (nx - freq_of(i, nx)) % nx;
        tcp[i + (size_t)nx * (j + (size_t)ny * k)] = tc[fx + (size_t)nx * (fy + (size_t)ny * fz)];
      }
    }
  }
  ND_CK(cudaMemcpy(p->d_tcp, tcp.data(), 8 * tcp.size(), cudaMemcpyHostToDevice));
  return ESPEC_OK;
}

extern "C" int espec_spond_energies(espec_spond_plan* p, double* e, double* norm, void* stream) {
  if (!p || !e || !norm) return set_error(ESPEC_EINVAL, "null argument");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_spond_load has not been called");
  cudaStream_t st = (cudaStream_t)stream;
  const long n = p->n;
  const int nb = 256;
  if (!p->d_khat) {
    ND_CK(cudaMalloc(&p->d_khat, sizeof(cpx<double>) * n));
    ND_CK(cudaMalloc(&p->d_tcp, 8 * n));
    ND_CK(cudaMalloc(&p->d_epart, sizeof(double2) * (nb + 1)));
    for (int ax = 0; ax < p->ndim; ++ax) {
      ND_CK(cudaMalloc(&p->d_tw64[ax], sizeof(RotD) * p->np[ax]));
      tw_table_kernel<double><<<(p->np[ax] + 255) / 256, 256, 0, st>>>(p->d_tw64[ax], p->np[ax]);
      ND_CK(cudaGetLastError());
    }
    const int rc = nd_energy_tables(p);
    if (rc) return rc;
  }
  NdArgs<double> a{};
  a.nx = p->np[0];
  a.ny = p->np[1];
  a.nz = p->ndim > 2 ? p->np[2] : 1;
  a.ndim = p->ndim;
  a.psi = p->d_khat;
  a.psi_start = p->has_state ? p->d_out : p->d_psi0;
  for (int ax = 0; ax < 3; ++ax) a.tw[ax] = ax < p->ndim ? p->d_tw64[ax] : nullptr;
  cudaError_t err = launch_x_n<double>(a.nx, kFwd0, a, p->xblocks, st);
  if (err == cudaSuccess)
    err = launch_axis<double>(a.ny, kFwd, false, a, 1, 0, st);
  if (err == cudaSuccess && p->ndim > 2)
    err = launch_axis<double>(a.nz, kFwd, false, a, 2, 0, st);
  if (err != cudaSuccess) return set_cuda_error("energy transform", err);
  nd_energy_kernel<<<nb, 256, 0, st>>>(a.psi_start, p->d_vpot, p->d_khat, p->d_tcp, n,
                                       1.0 / (double)n, p->d_epart);
  csum_kernel<<<1, 1, 0, st>>>(p->d_epart, nb, 0, 0, p->d_epart + nb);
  ND_CK(cudaGetLastError());
  double2 h;
  ND_CK(cudaMemcpyAsync(&h, p->d_epart + nb, sizeof h, cudaMemcpyDeviceToHost, st));
  ND_CK(cudaStreamSynchronize(st));
  *e = h.x;
  *norm = h.y;
  return ESPEC_OK;
}

extern "C" int espec_spond_results(espec_spond_plan* p, double* c_re, double* c_im,
                                   double* psi_re, double* psi_im, int where, void* stream) {
  if (!p || p->c_cap < 0) return set_error(ESPEC_EINVAL, "no results: run the plan first");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nc = (size_t)p->c_cap + 1, n = (size_t)p->n;
  int rc = get_complex(p->stage, p->d_c, c_re, c_im, nc, where, st);
  if (rc == ESPEC_OK) rc = get_complex(p->stage, p->d_out, psi_re, psi_im, n, where, st);
  if (rc) return rc;
  if (where == ESPEC_MEM_HOST) ND_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}

extern "C" void espec_spond_destroy(espec_spond_plan* p) {
  if (!p) return;
  void* b[] = {p->d_psi,    p->d_psi0,  p->d_out,   p->d_vpot,  p->d_vabc,   p->d_tab,
               p->d_kq,     p->d_cpart, p->d_c,     p->d_tw[0], p->d_tw[1],  p->d_tw[2],
               p->d_khat,   p->d_tcp,   p->d_epart, p->d_tw64[0], p->d_tw64[1], p->d_tw64[2],
               p->d_prev,   p->d_sod};
  for (void* x : b)
    if (x) cudaFree(x);
  p->stage.release();
  delete p;
}
