// sil.cu -- propagation on one grid (1D/2D/3D) with the finite-difference
// Hamiltonian, FP64: the short-iterative-Lanczos cooperative kernel described
// in sil.cuh, the second-order-differences kernel (.PSOD), the
// finite-difference energy kernel, and the grid plan behind espec_grid_*
// (include/espec_gpu.h).
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <utility>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"
#include "sil.cuh"

namespace espec {
namespace {

// a barrier wait gives up after this many polls (~ seconds); the kernel then
// sets the error flag and returns
constexpr long kSpinLimit = 1L << 24;

struct Range {
  int lo, hi;
};

__device__ __forceinline__ Range my_range(long n) {
  const long chunk = (n + gridDim.x - 1) / gridDim.x;
  long lo = (long)blockIdx.x * chunk, hi = lo + chunk;
  if (lo > n) lo = n;
  if (hi > n) hi = n;
  return Range{(int)lo, (int)hi};
}

// Loads of state that other CTAs wrote before the last grid barrier: plain
// loads.  The barrier's acquire (thread 0) and bar.sync order them after the
// writers' release, so the memory model gives them the written values; unlike
// the volatile __ldcg they leave the compiler free to issue several points'
// loads together.
__device__ __forceinline__ double ld_state(const double* p) { return *p; }

// Grid barrier fused with a reduction: sp[0..nq) holds this CTA's partial
// sums; on return st[0..nq) holds the totals over all CTAs.  After the
// barrier every CTA sums the G partials itself, in one fixed order, so all
// CTAs hold the same bits and no CTA waits for another's sum.  The partials
// alternate between two buffers by barrier parity (phase, counted alike by
// every thread of every CTA): a CTA runs at most one barrier ahead of the
// slowest, which can still be reading the other buffer.  false = a wait
// gave up.
template <int kInFlight = 16>
__device__ bool grid_reduce(const SilArgs& a, const double* sp, double* st, int nq,
                            int* s_flag, double* s_red /* kSilThreads doubles */,
                            unsigned& phase) {
  const int b = blockIdx.x, G = gridDim.x, t = threadIdx.x;
  if (G == 1) {  // one CTA: its partials are the totals (the same bits: 0 + x)
    ++phase;
    __syncthreads();
    for (int q = t; q < nq; q += blockDim.x) st[q] = 0.0 + sp[q];
    __syncthreads();
    return true;
  }
  double* part = a.part + (size_t)(phase & 1u) * G * kSilNQ;
  // a.bar counts the arrivals of the launch (zeroed before it): barrier k is
  // passed once it reaches (k + 1) G
  const unsigned long long target = (unsigned long long)(phase + 1u) * (unsigned)G;
  ++phase;
  // The CTA's writes are ordered before thread 0's arrival (a release RMW) by
  // bar.sync, whose ordering is cumulative; every arrival continues the
  // release sequence of the earlier ones, so a waiter's acquire load of the
  // final count synchronises with all of them.
  for (int q = t; q < nq; q += blockDim.x) part[(long)b * kSilNQ + q] = sp[q];
  __syncthreads();
  if (t == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> cnt(
        *reinterpret_cast<unsigned long long*>(a.bar));
    cuda::atomic_ref<int, cuda::thread_scope_device> err(*a.err);
    const unsigned long long arrived = cnt.fetch_add(1ull, cuda::memory_order_acq_rel) + 1ull;
    s_flag[1] = 1;
    if (arrived < target) {
      long spins = 0;
      while (cnt.load(cuda::memory_order_acquire) < target) {
        if (++spins > a.spin_limit || err.load(cuda::memory_order_relaxed) != 0) {
          err.store(1, cuda::memory_order_relaxed);
          s_flag[1] = 0;
          break;
        }
        if (spins > 4096) __nanosleep(32);
      }
    }
  }
  __syncthreads();
  if (!s_flag[1]) return false;
  // R threads per quantity, each summing every R-th CTA in CTA order with up
  // to kInFlight loads in flight (48: one round of L2 latency for 128 CTAs
  // and up to 96 quantities), then the R partial sums in order
  double* red = s_red;
  const int R = nq > 0 ? min(kSilThreads / nq, 32) : 1;
  if (t < R * nq) {
    const int q = t % nq, r = t / nq;
    double s = 0.0;
    for (int i0 = r; i0 < G; i0 += kInFlight * R) {
      double x[kInFlight];
#pragma unroll
      for (int j = 0; j < kInFlight; ++j) {
        const int i = i0 + j * R;
        x[j] = i < G ? __ldcg(part + (long)i * kSilNQ + q) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kInFlight; ++j) s += x[j];
    }
    red[r * nq + q] = s;
  }
  __syncthreads();
  for (int q = t; q < nq; q += blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < R; ++r) s += red[r * nq + q];
    st[q] = s;
  }
  __syncthreads();
  return true;
}

// sum of nv per-thread values over the CTA into sp[0..nv)
template <int NV>
__device__ __forceinline__ void block_sum(const double (&x)[NV], double* sp, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double s = x[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) scratch[warp * NV + i] = s;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < kSilThreads / 32; ++w) s += scratch[w * NV + threadIdx.x];
    sp[threadIdx.x] = s;
  }
  __syncthreads();
}

// (x, y, z) indices of point k on an NDIM grid, x fastest.  (k + 1/2)/nx
// by one FP64 multiplication: its rounding error (< k 2^-52) is far below the
// 1/(2 nx) distance to the nearest integer, so the truncation is exact.
template <int NDIM>
__device__ __forceinline__ void grid_index(const SilArgs& a, int k, int (&idx)[3]) {
  idx[1] = idx[2] = 0;
  if (NDIM == 1) {
    idx[0] = k;
  } else {
    const int q = (int)(((double)k + 0.5) * a.inv_nx);
    idx[0] = k - q * a.nx;
    if (NDIM == 2) {
      idx[1] = q;
    } else {
      const int z = (int)(((double)q + 0.5) * a.inv_ny);
      idx[1] = q - z * a.ny;
      idx[2] = z;
    }
  }
}

// H_FD x at point k of an NDIM grid, every x value scaled by d (au1d.f:52-73,
// au2di.f:57-225, au3d.f:61-117): (30 sum(shm) + V) x_k + sum_a shm_a
// (x_{-2} - 16 x_{-1} - 16 x_{+1} + x_{+2}), zero outside the grid; idx from
// grid_index.  Every neighbour load is issued unconditionally (from x_k where
// the neighbour is off the grid) so that no branch separates a point's loads
// from the next point's; the sums skip the off-grid terms.
template <int NDIM, typename T = double>
__device__ __forceinline__ T apply_h_nd(const SilArgs& a, const T* x, int k, T d,
                                        const int (&idx)[3]) {
  const int len[3] = {a.nx, a.ny, a.nz}, str[3] = {1, a.nx, a.nx * a.ny};
  T xm2[NDIM], xm1[NDIM], xp1[NDIM], xp2[NDIM];
#pragma unroll
  for (int ax = 0; ax < NDIM; ++ax) {
    const int i = idx[ax], st = str[ax], L = len[ax];
    xm2[ax] = x[i >= 2 ? k - 2 * st : k];
    xm1[ax] = x[i >= 1 ? k - st : k];
    xp1[ax] = x[i + 1 < L ? k + st : k];
    xp2[ax] = x[i + 2 < L ? k + 2 * st : k];
  }
  T s = ((T)a.sht30 + (T)__ldg(a.vpot + k)) * (x[k] * d);
#pragma unroll
  for (int ax = 0; ax < NDIM; ++ax) {
    const T h = (T)a.shm[ax];
    const int i = idx[ax], L = len[ax];
    if (i >= 2) s += h * (xm2[ax] * d);
    if (i >= 1) s += (T)-16.0 * h * (xm1[ax] * d);
    if (i + 1 < L) s += (T)-16.0 * h * (xp1[ax] * d);
    if (i + 2 < L) s += h * (xp2[ax] * d);
  }
  return s;
}

// Krylov coefficients of both chains (every CTA computes the same values):
// Z y = exp(-i cst T) y for the m x m symmetric tridiagonal T of each chain
// (diagonal al, off-diagonal bt), without forming Z: the Chebyshev series of
// the exponential on T's Gershgorin interval [c - h, c + h],
//   exp(-i tau T) y = e^{-i tau c} sum_k eps_k (-i)^k J_k(tau h) T_k((T - c)/h) y
// (eps_0 = 1, eps_k = 2; the Bessel values J_k by Miller's downward
// recurrence), i.e. one three-term vector recurrence with a tridiagonal
// product per term: one warp per series, lane i holding row i, no CTA
// barrier.  The series is cut where 2 |J_{K+1}| < 1e-17 (K = 1.5 tau h + 25
// terms, within kChebMax; a longer tau is split into equal parts applied in
// turn).  The reference forms the same matrix function through the
// eigenvectors of T (DSTEVX).  out[0] = Re Z y_u, out[1] = Im Z y_u (or
// Im(Z^2 y_u) / 2 in the reference-defect form, the series for 2 cst on a
// third warp), out[2] = Re Z y_v, out[3] = -Im Z y_v.
constexpr int kChebMax = 176;  // Bessel values kept per series

struct KrylovSmem {
  double J[3][kChebMax + 1];  // per series (warp)
};

// exp(-i tau T) y, row `lane` (m <= 32), by the whole warp; J: kChebMax + 1
// doubles of shared memory for this warp's Bessel values
__device__ double2 expm_tridiag_apply(int m, double tau, const double* al, const double* bt,
                                      const double* y, double* J) {
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  const bool row = lane < m;
  const double a_i = row ? al[lane] : 0.0;
  const double b_lo = (row && lane > 0) ? bt[lane - 1] : 0.0;  // T_{i,i-1}
  const double b_up = (row && lane + 1 < m) ? bt[lane] : 0.0;  // T_{i,i+1}
  // Gershgorin interval of T
  double lo = row ? a_i - fabs(b_lo) - fabs(b_up) : 1e300;
  double hi = row ? a_i + fabs(b_lo) + fabs(b_up) : -1e300;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(full, lo, o));
    hi = fmax(hi, __shfl_xor_sync(full, hi, o));
  }
  const double c = 0.5 * (lo + hi), h = 0.5 * (hi - lo);
  double xr = row ? y[lane] : 0.0, xi = 0.0;  // the vector the next part acts on
  if (h > 0.0) {
    const double za = fabs(tau) * h;
    const int parts = (int)ceil(za / 100.0) > 1 ? (int)ceil(za / 100.0) : 1;
    const double zp = za / parts;                    // |tau h| of one part
    const int K = min((int)(1.5 * zp) + 25, kChebMax);
    const double sgn = tau < 0.0 ? -1.0 : 1.0;       // J_k(-z) = (-1)^k J_k(z)
    if (lane == 0) {
      // Miller: J_{j-1} = (2j/z) J_j - J_{j+1} downward from a start 20
      // orders above K (J_K is already below 1e-17 of J_0 there), normalised
      // by J_0 + 2 sum_k J_2k = 1
      const int nstart = 2 * ((K + 21) / 2);
      const double tz = 2.0 / zp;
      double bjp = 0.0, bj = 1e-280, sum = 0.0, jd = nstart;
      for (int j = nstart; j > 0; --j, jd -= 1.0) {
        const double bjm = fma(jd * tz, bj, -bjp);
        bjp = bj;
        bj = bjm;
        if (fabs(bj) > 1e200) {
          bj *= 1e-200;
          bjp *= 1e-200;
          sum *= 1e-200;
          for (int k = j; k <= K; ++k) J[k] *= 1e-200;
        }
        if (j - 1 <= K) J[j - 1] = bj;
        if (((j - 1) & 1) == 0 && j - 1 > 0) sum += bj;
      }
      const double rn = 1.0 / (bj + 2.0 * sum);
      for (int k = 0; k <= K; ++k) J[k] *= ((k & 1) && sgn < 0.0 ? -rn : rn);
    }
    __syncwarp();
    const double rh = 1.0 / h;
    // (T - c)/h times v, row lane
    auto tmul = [&](double v) {
      const double vl = __shfl_up_sync(full, v, 1), vu = __shfl_down_sync(full, v, 1);
      return ((a_i - c) * v + b_lo * (lane > 0 ? vl : 0.0) + b_up * vu) * rh;
    };
    double sr, si;
    const double ph = -(tau / parts) * c;  // e^{-i (tau/parts) c}
    double ps, pc;
    sincos(ph, &ps, &pc);
    for (int part = 0; part < parts; ++part) {
      // real and imaginary parts of the input run through the same real
      // recurrence; (-i)^k cycles 1, -i, -1, i
      double w0r = xr, w0i = xi;
      double w1r = tmul(w0r), w1i = tmul(w0i);
      sr = J[0] * w0r;
      si = J[0] * w0i;
      // k = 1: -2i J_1 w1
      sr += 2.0 * J[1] * w1i;
      si -= 2.0 * J[1] * w1r;
      for (int k = 2; k <= K; ++k) {
        const double w2r = 2.0 * tmul(w1r) - w0r, w2i = 2.0 * tmul(w1i) - w0i;
        const double ck = 2.0 * J[k];
        switch (k & 3) {
          case 0: sr += ck * w2r; si += ck * w2i; break;
          case 1: sr += ck * w2i; si -= ck * w2r; break;
          case 2: sr -= ck * w2r; si -= ck * w2i; break;
          default: sr -= ck * w2i; si += ck * w2r; break;
        }
        w0r = w1r; w0i = w1i;
        w1r = w2r; w1i = w2i;
      }
      xr = pc * sr - ps * si;
      xi = pc * si + ps * sr;
    }
  } else {
    // T = c I (a 1 x 1 T or a zero off-diagonal with equal diagonal)
    double ps, pc;
    sincos(-tau * c, &ps, &pc);
    xi = ps * xr;
    xr = pc * xr;
  }
  return make_double2(xr, xi);
}

__device__ void krylov_coeffs(int m, double cst, int quirk, const double (*al)[kSilMaxM],
                              const double (*bt)[kSilMaxM], const double (*y)[kSilMaxM],
                              const int* active, KrylovSmem& ks, double (*out)[kSilMaxM]) {
  // warp 0: chain u, warp 1: chain v, warp 2: chain u over 2 cst (defect form)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w < 2 || (w == 2 && quirk)) {
    const int c = w == 1 ? 1 : 0;
    const double tau = w == 2 ? 2.0 * cst : cst;
    double2 z = make_double2(0.0, 0.0);
    if (active[c]) z = expm_tridiag_apply(m, tau, al[c], bt[c], y[c], ks.J[w]);
    if (lane < m) {
      if (w == 0) {
        out[0][lane] = z.x;
        if (!quirk) out[1][lane] = z.y;
      } else if (w == 1) {
        out[2][lane] = z.x;
        out[3][lane] = -z.y;
      } else {
        out[1][lane] = 0.5 * z.y;
      }
    }
  }
  __syncthreads();
}

}  // namespace

// per-chain slots of the partial sums of Lanczos iteration it:
//   it = 0: [<vi,H vi>, <vi,x>, <vi,vi>]
//   it > 0, res = the residual of iteration it-1 (unnormalised), vp = that
//   iteration's vector: [<res,H res>, <res,x>, <res,res>, <H res,L_q> (q < it),
//   <res,L_q> (q < it), <vp,L_q> (q < it)]
__device__ __forceinline__ int nslots(int it) { return 3 + 3 * it; }
__device__ __forceinline__ int slot_of(int c, int it, int i) { return c * nslots(it) + i; }

// warp sum of x into ws[warp][slot] (called by the whole CTA alike)
__device__ __forceinline__ void warp_put(double x, int slot, double* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if (lane == 0) ws[warp * kSilNQ + slot] = x;
}

// Warp reduce-scatter of V values per lane (V = 16 or 32): returns, in lane
// l, the warp's sum of value l (V = 32) or of value l & 15 (V = 16).  Each
// round sends half of the values still held to the partner lane and keeps
// the other half: V - 1 shuffles in all, against five per value for
// one-value-at-a-time sums.
template <int V>
__device__ __forceinline__ double warp_scatter(double (&x)[V]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int half = V / 2; half >= 1; half >>= 1) {
    const bool up = (lane & half) != 0;
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const double give = up ? x[j] : x[j + half];
      const double keep = up ? x[j + half] : x[j];
      x[j] = keep + __shfl_xor_sync(0xffffffffu, give, half);
    }
  }
  double r = x[0];
  if (V == 16) r += __shfl_xor_sync(0xffffffffu, r, 16);
  return r;
}

// Neighbour handshake of a pass whose results other CTAs' stencils read:
// after this CTA's writes it publishes epoch ep in its flag (a release after
// bar.sync, as in grid_reduce), then waits until every CTA owning a point
// within `reach` of its own range has published ep (acquire loads; flags are
// zeroed before the launch and grow by one per handshake, and no CTA can be a
// whole handshake ahead: the grid reduction between two handshakes waits for
// all).  false = a wait gave up (error flag set).
__device__ bool halo_sync(const SilArgs& a, Range r, long reach, unsigned ep) {
  const int b = blockIdx.x, G = gridDim.x, t = threadIdx.x;
  __syncthreads();
  if (t == 0) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> f(a.nflag[b]);
    f.store(ep, cuda::memory_order_release);
  }
  bool ok = true;
  if (r.lo < r.hi) {
    const long chunk = (a.n + G - 1) / G;
    const long lo = r.lo - reach > 0 ? r.lo - reach : 0;
    const long hi = r.hi - 1 + reach < a.n - 1 ? r.hi - 1 + reach : a.n - 1;
    const int first = (int)(lo / chunk), last = (int)(hi / chunk);
    cuda::atomic_ref<int, cuda::thread_scope_device> err(*a.err);
    for (int j = first + t; j <= last && ok; j += blockDim.x) {
      if (j == b) continue;
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> f(a.nflag[j]);
      long spins = 0;
      while (f.load(cuda::memory_order_acquire) < ep) {
        if (++spins > a.spin_limit || err.load(cuda::memory_order_relaxed) != 0) {
          err.store(1, cuda::memory_order_relaxed);
          ok = false;
          break;
        }
        if (spins > 4096) __nanosleep(32);
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

// Where a step's Lanczos vectors, its H residual and the CTA's copy of its
// residual live.  All three are read at the CTA's own points only, so with
// kS they stay in the CTA's shared memory ([2][m][chunk] vectors, [2][chunk]
// H residual, [2][chunk] residual; kl = point - first point of the CTA) and
// the vectors reach global memory in the launch's last step only (the
// drop-ins return that basis).  The residual is also written to global
// memory: the neighbouring CTAs' stencils read it there.
template <bool kS, typename S>
struct SilVecs {
  S* L;   // global [2][m][n]
  S* wb;  // global [2][n]
  S* wk;  // global [2][n]
  S* sm;  // shared (kS)
  long n;
  int m, chunk;
  __device__ __forceinline__ double l(int c, int q, int k, int kl) const {
    if constexpr (kS) return (double)sm[((long)c * m + q) * chunk + kl];
    else return (double)L[((long)c * m + q) * n + k];
  }
  __device__ __forceinline__ void set_l(int c, int q, int k, int kl, double v) const {
    if constexpr (kS) sm[((long)c * m + q) * chunk + kl] = (S)v;
    else L[((long)c * m + q) * n + k] = (S)v;
  }
  __device__ __forceinline__ double w(int c, int k, int kl) const {
    if constexpr (kS) return (double)sm[(long)(2 * m + c) * chunk + kl];
    else return (double)wb[(long)c * n + k];
  }
  __device__ __forceinline__ void set_w(int c, int k, int kl, double v) const {
    if constexpr (kS) sm[(long)(2 * m + c) * chunk + kl] = (S)v;
    else wb[(long)c * n + k] = (S)v;
  }
  __device__ __forceinline__ double res(int c, int k, int kl) const {
    if constexpr (kS) return (double)sm[(long)(2 * m + 2 + c) * chunk + kl];
    else return (double)wk[(long)c * n + k];
  }
  __device__ __forceinline__ void set_res(int c, int k, int kl, double v) const {
    if constexpr (kS) sm[(long)(2 * m + 2 + c) * chunk + kl] = (S)v;
    wk[(long)c * n + k] = (S)v;
  }
};

// dynamic shared memory of the kS form for m vectors and chunk points per
// CTA, vectors of `bytes` bytes per value
__host__ __device__ constexpr size_t sil_vec_smem(int m, long chunk, int bytes) {
  return (size_t)(2 * m + 4) * (size_t)chunk * (size_t)bytes;
}

// S: the storage (and stencil arithmetic) of the Lanczos vectors, the
// residual and H times the residual -- double, or float in the mixed form
// (dot products, coefficients, Krylov exponential and state in FP64 both ways)
template <int NDIM, bool kS, typename S>
__global__ void __launch_bounds__(kSilThreads, 1) sil_kernel(SilArgs a) {
  extern __shared__ __align__(16) unsigned char sil_dyn_raw[];
  S* sil_dyn = reinterpret_cast<S*>(sil_dyn_raw);
  __shared__ double sp[kSilNQ], st[kSilNQ], scratch[(kSilThreads / 32) * 8];
  __shared__ double ws[(kSilThreads / 32) * kSilNQ];
  __shared__ double s_red[kSilThreads];
  __shared__ int s_flag[2];
  __shared__ double s_al[2][kSilMaxM], s_bt[2][kSilMaxM], s_proj[2][kSilMaxM];
  __shared__ double s_rbt[2][kSilMaxM];  // 1/bt, the scale of the next vector
  __shared__ double s_r[2][kSilMaxM], s_coef[4][kSilMaxM];
  __shared__ double s_bt0[2];
  __shared__ int s_active[2];
  __shared__ KrylovSmem ks;
  const Range r = my_range(a.n);
  const int t = threadIdx.x;
  const long n = a.n;
  const int m = a.m;
  SilVecs<kS, S> vs;
  vs.L = reinterpret_cast<S*>(a.L);
  vs.wb = reinterpret_cast<S*>(a.wbuf);
  vs.wk = reinterpret_cast<S*>(a.work);
  vs.sm = sil_dyn;
  vs.n = n;
  vs.m = m;
  vs.chunk = (int)((n + gridDim.x - 1) / gridDim.x);
  unsigned phase = 0;  // grid barriers passed in this launch
  unsigned hep = 0;    // neighbour handshakes passed in this launch
  constexpr int NW = kSilThreads / 32;
  // farthest point the 4th-order stencil reads: two lines of the slowest axis
  const long reach = 2L * (NDIM == 1 ? 1L : NDIM == 2 ? (long)a.nx : (long)a.nx * a.ny);

  // this thread's sums for the norms of u, v and C of the state it wrote last
  // (the expansion below accumulates them for the next step, in the same
  // point order as the loop here)
  double qn[6] = {0, 0, 0, 0, 0, 0};
  for (int s = 0;; ++s) {
    // ---- norms of u, v and C(s) = <psi0|psi(s)> (pspofft.f:119-120 form)
    {
      double q[6] = {0, 0, 0, 0, 0, 0};
      if (s == 0) {
        for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
          const double uk = ld_state(a.u + k), vk = ld_state(a.v + k);
          const double u0k = __ldg(a.u0 + k), v0k = __ldg(a.v0 + k);
          q[0] += uk * uk;
          q[1] += vk * vk;
          q[2] += u0k * uk;
          q[3] += v0k * vk;
          q[4] += u0k * vk;
          q[5] += v0k * uk;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) q[i] = qn[i];
      }
      block_sum<6>(q, sp, scratch);
      if (!grid_reduce<48>(a, sp, st, 6, s_flag, s_red, phase)) return;
      if (t == 0 && blockIdx.x == 0 && (s > 0 || a.write_c0))
        a.c_out[s] = make_double2(st[2] + st[3], st[4] - st[5]);
      if (s == a.nsteps) break;
      if (t < 2) {
        s_bt0[t] = sqrt(st[t]);
        s_active[t] = st[t] != 0.0;  // lnz.f:88 (BT0.EQ.0: no Lanczos vectors)
      }
      __syncthreads();
    }
    // potential of this step with a pulse (pplnz.f:139-141): V - DM EF(T) of
    // the time the step lands at
    const double efs = a.dm ? a.ef[a.slot0 + s + 1] : 0.0;
    // ---- m Lanczos iterations of both chains, one grid-wide reduction each
    for (int it = 0; it < m; ++it) {
      if (it == 0) {
        // vi = x/bt0 and w = H vi at the CTA's points; <vi,w>, <vi,x>, <vi,vi>
        for (int c = 0; c < 2; ++c) {
          const double bt0 = s_bt0[c];
          // vi = x * (1/bt0) here and for the stencil's neighbours alike, so
          // the stencil sees exactly the stored vi
          const double rb = 1.0 / bt0;
          const double* x = c ? a.v : a.u;
          double acc[3] = {0.0, 0.0, 0.0};
          if (s_active[c]) {
            auto point = [&](int k, double& vi_out, double& w_out) __attribute__((always_inline)) {
              const double xk = ld_state(x + k);
              const double vi = xk * rb;
              int idx[3];
              grid_index<NDIM>(a, k, idx);
              double hv = apply_h_nd<NDIM>(a, x, k, rb, idx);
              if (a.dm) hv -= __ldg(a.dm + k) * efs * vi;
              vi_out = vi;
              w_out = hv;  // no previous vector: w = H vi
              acc[0] += vi * hv;
              acc[1] += vi * xk;
              acc[2] += vi * vi;
            };
            int k0 = r.lo + t;
            for (; k0 + kSilThreads < r.hi; k0 += 2 * kSilThreads) {
              double vi0, w0, vi1, w1;
              point(k0, vi0, w0);
              point(k0 + kSilThreads, vi1, w1);
              vs.set_l(c, 0, k0, k0 - r.lo, vi0);
              vs.set_w(c, k0, k0 - r.lo, w0);
              vs.set_l(c, 0, k0 + kSilThreads, k0 + kSilThreads - r.lo, vi1);
              vs.set_w(c, k0 + kSilThreads, k0 + kSilThreads - r.lo, w1);
            }
            for (; k0 < r.hi; k0 += kSilThreads) {
              double vi0, w0;
              point(k0, vi0, w0);
              vs.set_l(c, 0, k0, k0 - r.lo, vi0);
              vs.set_w(c, k0, k0 - r.lo, w0);
            }
          } else {
            for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
              vs.set_l(c, 0, k, k - r.lo, 0.0);
              vs.set_w(c, k, k - r.lo, 0.0);
            }
          }
#pragma unroll
          for (int i = 0; i < 3; ++i) warp_put(acc[i], slot_of(c, 0, i), ws);
        }
      } else {
        // pass 1: the residual of iteration p = it - 1 at the CTA's points
        // (lnz.f / reort.f: work = w - al vi - sum_q r_q L_q); vi_p and w_p
        // from the previous pass's unnormalised residual and H residual:
        // vi_p = res * (1/bt), w_p = (H res) * (1/bt) - bt vi_{p-1}
        const int p = it - 1;
        // per chain: [0] <res,res>, [1 + q] <vi_p, L_q> (q <= p <= 14)
        double acc1[2][16];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int i = 0; i < 16; ++i) acc1[c][i] = 0.0;
        // two points x two chains per thread at a time, the Gram-Schmidt
        // sum of each as its own chain of operations (q outermost), so that
        // the four interleave
        for (int k0 = r.lo + t; k0 < r.hi; k0 += 2 * kSilThreads) {
          const int kk[2] = {k0, k0 + kSilThreads};
          bool on[2][2];
          double vi[2][2], res[2][2];
#pragma unroll
          for (int pt = 0; pt < 2; ++pt)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int k = kk[pt], kl = k - r.lo;
              on[pt][c] = k < r.hi && s_active[c];
              vi[pt][c] = res[pt][c] = 0.0;
              if (on[pt][c]) {
                double w;
                if (p == 0) {
                  vi[pt][c] = vs.l(c, 0, k, kl);
                  w = vs.w(c, k, kl);
                } else {
                  const double bp = s_bt[c][p - 1], rbp = s_rbt[c][p - 1];
                  vi[pt][c] = vs.res(c, k, kl) * rbp;
                  w = vs.w(c, k, kl) * rbp - bp * vs.l(c, p - 1, k, kl);
                }
                res[pt][c] = w - s_al[c][p] * vi[pt][c];
              }
            }
#pragma unroll
          for (int q = 0; q < 15; ++q) {
            if (q < p) {
#pragma unroll
              for (int pt = 0; pt < 2; ++pt)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                  if (on[pt][c]) {
                    const double lq = vs.l(c, q, kk[pt], kk[pt] - r.lo);
                    res[pt][c] -= s_r[c][q] * lq;
                    acc1[c][1 + q] += vi[pt][c] * lq;
                  }
            }
          }
#pragma unroll
          for (int pt = 0; pt < 2; ++pt)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int k = kk[pt], kl = k - r.lo;
              if (k >= r.hi) continue;
              if (on[pt][c]) {
                res[pt][c] -= s_r[c][p] * vi[pt][c];
                acc1[c][0] += res[pt][c] * res[pt][c];
#pragma unroll
                for (int q = 0; q < 15; ++q)
                  if (q == p) acc1[c][1 + q] += vi[pt][c] * vi[pt][c];
              }
              if (p >= 1) vs.set_l(c, p, k, kl, vi[pt][c]);
              vs.set_res(c, k, kl, res[pt][c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const double v = warp_scatter<16>(acc1[c]);
          const int lane = t & 31, i = lane;
          if (i == 0) ws[(t >> 5) * kSilNQ + slot_of(c, it, 2)] = v;
          else if (i <= it) ws[(t >> 5) * kSilNQ + slot_of(c, it, 3 + 2 * it + i - 1)] = v;
        }
        // the residual at the points this CTA's stencil reaches is written
        if (!halo_sync(a, r, reach, ++hep)) return;
        // pass 2: H res at the CTA's points and the unnormalised dot products
        // of iteration it: <res,H res>, <res,x>, <H res,L_q>, <res,L_q>.
        // First the stencils (global loads of the neighbours' residual) of
        // two points x two chains together, H res kept with the CTA's
        // vectors; then the products against the vectors.
        double dd[2][2] = {{0.0, 0.0}, {0.0, 0.0}};  // [c]: <res,H res>, <res,x>
        for (int k0 = r.lo + t; k0 < r.hi; k0 += 2 * kSilThreads) {
          const int kk[2] = {k0, k0 + kSilThreads};
          double hr[2][2], rk[2][2], xk[2][2];
#pragma unroll
          for (int pt = 0; pt < 2; ++pt)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int k = kk[pt];
              hr[pt][c] = rk[pt][c] = xk[pt][c] = 0.0;
              if (k < r.hi && s_active[c]) {
                const S* rc = vs.wk + (long)c * n;
                int idx[3];
                grid_index<NDIM>(a, k, idx);
                rk[pt][c] = vs.res(c, k, k - r.lo);
                hr[pt][c] = (double)apply_h_nd<NDIM, S>(a, rc, k, (S)1, idx);
                if (a.dm) hr[pt][c] -= __ldg(a.dm + k) * efs * rk[pt][c];
                xk[pt][c] = ld_state((c ? a.v : a.u) + k);
              }
            }
#pragma unroll
          for (int pt = 0; pt < 2; ++pt)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int k = kk[pt];
              if (k < r.hi && s_active[c]) {
                vs.set_w(c, k, k - r.lo, hr[pt][c]);
                dd[c][0] += rk[pt][c] * hr[pt][c];
                dd[c][1] += rk[pt][c] * xk[pt][c];
              }
            }
        }
        for (int c = 0; c < 2; ++c) {
          // [0] <res,H res>, [1] <res,x>, [2 + q] <H res,L_q>, [17 + q] <res,L_q>
          // (q < it <= 15)
          double acc[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[i] = 0.0;
          acc[0] = dd[c][0];
          acc[1] = dd[c][1];
          if (s_active[c]) {
            for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
              const int kl = k - r.lo;
              const double hk = vs.w(c, k, kl), rq = vs.res(c, k, kl);
#pragma unroll
              for (int q = 0; q < 15; ++q) {
                if (q < it) {
                  const double lq = vs.l(c, q, k, kl);
                  acc[2 + q] += hk * lq;
                  acc[17 + q] += rq * lq;
                }
              }
            }
          }
          const double v = warp_scatter<32>(acc);
          const int i = t & 31;
          int slot = -1;
          if (i < 2) slot = slot_of(c, it, i);
          else if (i < 17) slot = i - 2 < it ? slot_of(c, it, 3 + i - 2) : -1;
          else slot = i - 17 < it ? slot_of(c, it, 3 + it + i - 17) : -1;
          if (slot >= 0) ws[(t >> 5) * kSilNQ + slot] = v;
        }
      }
      __syncthreads();
      const int nq = 2 * nslots(it);
      for (int q = t; q < nq; q += kSilThreads) {
        double sum = 0.0;
        for (int w = 0; w < NW; ++w) sum += ws[w * kSilNQ + q];
        sp[q] = sum;
      }
      __syncthreads();
      if (!grid_reduce<48>(a, sp, st, nq, s_flag, s_red, phase)) return;
      // the iteration's coefficients: thread (c, q) of the first two warps
      // forms r_q of chain c; every one of them forms bt and al alike
      if (t < 64 && (t & 31) <= it) {
        const int c = t >> 5, q = t & 31, b0 = slot_of(c, it, 0);
        if (!s_active[c]) {
          s_r[c][q] = 0.0;
          if (q == 0) {
            s_al[c][it] = s_proj[c][it] = 0.0;
            if (it > 0) s_bt[c][it - 1] = s_rbt[c][it - 1] = 0.0;
          }
        } else if (it == 0) {
          const double al = st[b0];
          s_al[c][0] = al;
          s_proj[c][0] = st[b0 + 1];
          s_r[c][0] = al - al * st[b0 + 2];  // reort.f against vi itself
        } else {
          // bt = |res| of iteration it-1 (lnz.f:113); vi = res/bt and
          // w = H res/bt - bt vi_{it-1}, so al = <res,H res>/bt^2 -
          // <res,vi_{it-1}>, <w,L_q> = <H res,L_q>/bt - bt <vi_{it-1},L_q>,
          // <vi,L_q> = <res,L_q>/bt
          const double bt = sqrt(st[b0 + 2]);
          const double rb = 1.0 / bt;
          const double al = st[b0] * rb * rb - st[b0 + 3 + it + (it - 1)];
          if (q < it) {
            const double wl = st[b0 + 3 + q] * rb - bt * st[b0 + 3 + 2 * it + q];
            s_r[c][q] = wl - al * (st[b0 + 3 + it + q] * rb);
          } else {
            s_r[c][it] = al - al * (st[b0 + 2] * rb * rb);
            s_bt[c][it - 1] = bt;
            s_rbt[c][it - 1] = rb;
            s_al[c][it] = al;
            s_proj[c][it] = st[b0 + 1] * rb;
          }
        }
      }
      __syncthreads();
    }
    // ---- Krylov exponential and the new state
    krylov_coeffs(m, a.cst, a.quirk, s_al, s_bt, s_proj, s_active, ks, s_coef);
    // the last Lanczos vector is formed here: vi_{m-1} = res * (1/bt) from the
    // residual of iteration m-2 (an inactive chain's residual is zero), and
    // stored with the others (the drop-ins return the step's basis)
    const int ms = m >= 2 ? m - 1 : m;  // vectors stored by the iterations
    const double rbu = (m >= 2 && s_active[0]) ? s_rbt[0][m - 2] : 0.0;
    const double rbv = (m >= 2 && s_active[1]) ? s_rbt[1][m - 2] : 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) qn[i] = 0.0;
    // the launch's last step leaves its basis in global memory
    const bool basis_out = kS && s == a.nsteps - 1;
    for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
      const int kl = k - r.lo;
      double lu[kSilMaxM], lv[kSilMaxM];
#pragma unroll
      for (int j = 0; j < kSilMaxM; ++j) {
        lu[j] = j < ms ? vs.l(0, j, k, kl) : (j < m ? vs.res(0, k, kl) * rbu : 0.0);
        lv[j] = j < ms ? vs.l(1, j, k, kl) : (j < m ? vs.res(1, k, kl) * rbv : 0.0);
      }
      if (basis_out) {
#pragma unroll
        for (int j = 0; j < kSilMaxM; ++j)
          if (j < m) {
            vs.L[(long)j * n + k] = (S)lu[j];
            vs.L[(long)(m + j) * n + k] = (S)lv[j];
          }
      } else if (!kS && ms < m) {
#pragma unroll
        for (int j = 0; j < kSilMaxM; ++j)
          if (j == ms) {
            vs.L[(long)j * n + k] = (S)lu[j];
            vs.L[(long)(m + j) * n + k] = (S)lv[j];
          }
      }
      double ur = 0.0, ui = 0.0, vr = 0.0, vi = 0.0;
#pragma unroll
      for (int j = 0; j < kSilMaxM; ++j) {
        if (j < m) {
          ur += lu[j] * s_coef[0][j];
          ui += lu[j] * s_coef[1][j];
          vi += lv[j] * s_coef[2][j];
          vr += lv[j] * s_coef[3][j];
        }
      }
      double un = ur + vr, vn = ui + vi;
      if (a.mask) {  // sil.f:171-175
        const double mk = __ldg(a.mask + k);
        un = mk * un;
        vn = mk * vn;
      }
      a.u[k] = un;
      a.v[k] = vn;
      const double u0k = __ldg(a.u0 + k), v0k = __ldg(a.v0 + k);
      qn[0] += un * un;
      qn[1] += vn * vn;
      qn[2] += u0k * un;
      qn[3] += v0k * vn;
      qn[4] += u0k * vn;
      qn[5] += v0k * un;
    }
    __syncthreads();
  }
}

// points per thread whose loads are in flight together: four in 1D/2D, two in
// 3D (its 13-point stencils), within 128 registers
template <int NDIM>
constexpr int kPsodIlp = NDIM == 3 ? 2 : 4;

template <int KABS, bool DM, int NDIM>
__device__ __forceinline__ void psod_points(const SilArgs& a, Range r, const double* un,
                                            const double* vn, double* um, double* vm, double c,
                                            double e, double (&q)[4]);

// PSOD on a 2D grid by column strips: CTA b owns columns [256 s, 256 s + 256)
// (s = b mod nstrips) of a band of rows; each thread walks its column down the
// band with the y-stencil's five rows of psi_n in registers, so psi_n is read
// from memory once per band (plus two halo rows at each end), the x
// neighbours come from the row the warp has just loaded (L1), and every other
// array is one streaming read or write per point.
constexpr int kBandMinRows = 16;

struct Band {
  int col, r0, r1;
};

__device__ __forceinline__ Band my_band(const SilArgs& a) {
  const int ns = a.nstrips, nb = gridDim.x / ns;
  const int s = blockIdx.x % ns, band = blockIdx.x / ns;
  const int rows = (a.ny + nb - 1) / nb;
  Band B;
  B.col = s * kSilThreads + threadIdx.x;
  B.r0 = min(band * rows, a.ny);
  B.r1 = min(B.r0 + rows, a.ny);
  return B;
}

// (psi_n and psi_{n-1} are distinct buffers within a step: the loads of later
// rows may move ahead of this row's stores)
template <int KABS, bool DM>
__device__ __forceinline__ void psod2d_band(const SilArgs& a, const Band& B,
                                            const double* __restrict__ un,
                                            const double* __restrict__ vn,
                                            double* __restrict__ um, double* __restrict__ vm,
                                            double c, double e, double (&q)[4]) {
  const int nx = a.nx, ny = a.ny, col = B.col;
  if (col >= nx || B.r0 >= B.r1) return;
  const double hx = a.shm[0], hy = a.shm[1];
  // rows r-2 .. r+2 of psi_n at this column (zero off the grid)
  double wu[5], wv[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const int row = B.r0 - 2 + j;
    const bool in = row >= 0 && row < ny;
    wu[j] = in ? ld_state(un + (long)row * nx + col) : 0.0;
    wv[j] = in ? ld_state(vn + (long)row * nx + col) : 0.0;
  }
#pragma unroll 4
  for (int r = B.r0; r < B.r1; ++r) {
    const long k = (long)r * nx + col;
    // x neighbours of row r, issued unconditionally (from k when off the grid)
    const long xm2 = col >= 2 ? k - 2 : k, xm1 = col >= 1 ? k - 1 : k;
    const long xp1 = col + 1 < nx ? k + 1 : k, xp2 = col + 2 < nx ? k + 2 : k;
    const double um2 = ld_state(un + xm2), um1 = ld_state(un + xm1);
    const double up1 = ld_state(un + xp1), up2 = ld_state(un + xp2);
    const double vm2 = ld_state(vn + xm2), vm1 = ld_state(vn + xm1);
    const double vp1 = ld_state(vn + xp1), vp2 = ld_state(vn + xp2);
    const double vk = __ldg(a.vpot + k);
    const double umk = um[k], vmk = vm[k];
    const double u0k = __ldg(a.u0 + k), v0k = __ldg(a.v0 + k);
    // the next window row
    const int rn = r + 3;
    const bool inn = rn < ny;
    const double nu3 = inn ? ld_state(un + (long)rn * nx + col) : 0.0;
    const double nv3 = inn ? ld_state(vn + (long)rn * nx + col) : 0.0;
    // H psi_n at (col, r): au2di.f's terms in apply_h_nd's order
    double hu = (a.sht30 + vk) * wu[2], hv = (a.sht30 + vk) * wv[2];
    if (col >= 2) { hu += hx * um2; hv += hx * vm2; }
    if (col >= 1) { hu += -16.0 * hx * um1; hv += -16.0 * hx * vm1; }
    if (col + 1 < nx) { hu += -16.0 * hx * up1; hv += -16.0 * hx * vp1; }
    if (col + 2 < nx) { hu += hx * up2; hv += hx * vp2; }
    if (r >= 2) { hu += hy * wu[0]; hv += hy * wv[0]; }
    if (r >= 1) { hu += -16.0 * hy * wu[1]; hv += -16.0 * hy * wv[1]; }
    if (r + 1 < ny) { hu += -16.0 * hy * wu[3]; hv += -16.0 * hy * wv[3]; }
    if (r + 2 < ny) { hu += hy * wu[4]; hv += hy * wv[4]; }
    const double uk = wu[2], vkk = wv[2];
    if (DM) {
      const double de = __ldg(a.dm + k) * e;
      hv -= de * vkk;
      hu -= de * uk;
    }
    double nu, nv;
    if (KABS == 1) {
      const double w = a.vabc[k];
      nu = umk + c * hv - c * w * uk;
      nv = vmk - c * hu - c * w * vkk;
    } else if (KABS == 2) {
      const double w = a.vabc[k];
      nu = w * (umk + c * hv);
      nv = w * (vmk - c * hu);
    } else {
      nu = umk + c * hv;
      nv = vmk - c * hu;
    }
    um[k] = nu;
    vm[k] = nv;
    q[0] += u0k * nu;
    q[1] += v0k * nv;
    q[2] += u0k * nv;
    q[3] += v0k * nu;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      wu[j] = wu[j + 1];
      wv[j] = wv[j + 1];
    }
    wu[4] = nu3;
    wv[4] = nv3;
  }
}

template <int NDIM>
__device__ __forceinline__ void psod_dispatch(const SilArgs& a, Range r, const double* un,
                                              const double* vn, double* um, double* vm, double c,
                                              double e, double (&q)[4]) {
  if (NDIM == 2 && a.nstrips > 0) {
    const Band B = my_band(a);
    switch (a.kabs + (a.dm ? 3 : 0)) {
      case 0: psod2d_band<0, false>(a, B, un, vn, um, vm, c, e, q); break;
      case 1: psod2d_band<1, false>(a, B, un, vn, um, vm, c, e, q); break;
      case 2: psod2d_band<2, false>(a, B, un, vn, um, vm, c, e, q); break;
      case 3: psod2d_band<0, true>(a, B, un, vn, um, vm, c, e, q); break;
      case 4: psod2d_band<1, true>(a, B, un, vn, um, vm, c, e, q); break;
      default: psod2d_band<2, true>(a, B, un, vn, um, vm, c, e, q); break;
    }
    return;
  }
  switch (a.kabs + (a.dm ? 3 : 0)) {
    case 0: psod_points<0, false, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
    case 1: psod_points<1, false, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
    case 2: psod_points<2, false, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
    case 3: psod_points<0, true, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
    case 4: psod_points<1, true, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
    default: psod_points<2, true, NDIM>(a, r, un, vn, um, vm, c, e, q); break;
  }
}

// psi_{n-1}(k) <- psi_{n-1}(k) - i c H psi_n(k) with absorber KABS (0 none,
// 1 .VOPTIC, 2 .SMOOTHW) and, with DM, the field term; returns the new value
template <int KABS, bool DM, int NDIM>
__device__ __forceinline__ void psod_point(const SilArgs& a, const double* un, const double* vn,
                                           const double* um, const double* vm, int k, double c,
                                           double e, double& nu, double& nv) {
  const double uk = ld_state(un + k), vk = ld_state(vn + k);
  int idx[3];
  grid_index<NDIM>(a, k, idx);
  double hv = apply_h_nd<NDIM>(a, vn, k, 1.0, idx), hu = apply_h_nd<NDIM>(a, un, k, 1.0, idx);
  if (DM) {
    const double de = __ldg(a.dm + k) * e;
    hv -= de * vk;
    hu -= de * uk;
  }
  if (KABS == 1) {
    const double w = a.vabc[k];
    nu = um[k] + c * hv - c * w * uk;
    nv = vm[k] - c * hu - c * w * vk;
  } else if (KABS == 2) {
    const double w = a.vabc[k];
    nu = w * (um[k] + c * hv);
    nv = w * (vm[k] - c * hu);
  } else {
    nu = um[k] + c * hv;
    nv = vm[k] - c * hu;
  }
}

// one PSOD step over the CTA's points, kPsodIlp points per thread at a time
// with all their loads issued before the first store (no branch between
// them), then the rest one by one; q gets <psi0|psi_{n+1}>'s four sums in
// point order
template <int KABS, bool DM, int NDIM>
__device__ __forceinline__ void psod_points(const SilArgs& a, Range r, const double* un,
                                            const double* vn, double* um, double* vm, double c,
                                            double e, double (&q)[4]) {
  const int t = threadIdx.x;
  int k0 = r.lo + t;
  for (; k0 + (kPsodIlp<NDIM> - 1) * kSilThreads < r.hi; k0 += kPsodIlp<NDIM> * kSilThreads) {
    double nu[kPsodIlp<NDIM>], nv[kPsodIlp<NDIM>], u0k[kPsodIlp<NDIM>], v0k[kPsodIlp<NDIM>];
#pragma unroll
    for (int j = 0; j < kPsodIlp<NDIM>; ++j) {
      const int k = k0 + j * kSilThreads;
      psod_point<KABS, DM, NDIM>(a, un, vn, um, vm, k, c, e, nu[j], nv[j]);
      u0k[j] = __ldg(a.u0 + k);
      v0k[j] = __ldg(a.v0 + k);
    }
#pragma unroll
    for (int j = 0; j < kPsodIlp<NDIM>; ++j) {
      const int k = k0 + j * kSilThreads;
      um[k] = nu[j];
      vm[k] = nv[j];
      q[0] += u0k[j] * nu[j];
      q[1] += v0k[j] * nv[j];
      q[2] += u0k[j] * nv[j];
      q[3] += v0k[j] * nu[j];
    }
  }
  for (; k0 < r.hi; k0 += kSilThreads) {
    double nu, nv;
    psod_point<KABS, DM, NDIM>(a, un, vn, um, vm, k0, c, e, nu, nv);
    const double u0k = __ldg(a.u0 + k0), v0k = __ldg(a.v0 + k0);
    um[k0] = nu;
    vm[k0] = nv;
    q[0] += u0k * nu;
    q[1] += v0k * nv;
    q[2] += u0k * nv;
    q[3] += v0k * nu;
  }
}

// Second-order differences with H = AU (psod.f:64-205, sod.f:64-123), one
// cooperative kernel per run.  Each step overwrites the state one step back
// in place, psi_{n-1} <- psi_{n-1} - i c H psi_n (.VOPTIC: - c VABC psi_n;
// .SMOOTHW: the whole right side times the mask), reads psi_n's neighbours
// only, and ends in one grid barrier that also sums C = <psi0|psi_{n+1}>;
// then the two buffers swap roles.  From the start: C(0), an Euler step of
// c = CST/4 and a midpoint step of CST/2 to TI + DT, psi_{n-1} reset to psi0
// (with the reference's copy defect on request), then steps of CST.
//
// Two CTAs per SM (128 registers, no spills): the passes over a large grid are
// load-latency bound, and more warps hide it.
template <int NDIM>
__global__ void __launch_bounds__(kSilThreads, 2) psod_kernel(SilArgs a) {
  __shared__ double sp[4], st[4], scratch[(kSilThreads / 32) * 8];
  __shared__ double s_red[kSilThreads];
  __shared__ int s_flag[2];
  const Range r = my_range(a.n);
  const int t = threadIdx.x;
  unsigned phase = 0;  // grid barriers passed in this launch
  double *un = a.u, *vn = a.v, *um = a.up, *vm = a.vp;
  auto reduce_c = [&](double (&q)[4], int slot) -> bool {
    block_sum<4>(q, sp, scratch);
    if (!grid_reduce(a, sp, st, 4, s_flag, s_red, phase)) return false;
    if (t == 0 && blockIdx.x == 0 && slot >= 0)
      a.c_out[slot] = make_double2(st[0] + st[1], st[2] - st[3]);
    return true;
  };
  auto step = [&](double c, int slot, long call) __attribute__((always_inline)) -> bool {
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const double e = a.ef ? a.ef[call] : 0.0;  // chpot.f:46-50: V - DM EF
    // the absorber, the field and the dimension as template arguments
    psod_dispatch<NDIM>(a, r, un, vn, um, vm, c, e, q);
    if (!reduce_c(q, slot)) return false;
    double* x = un;
    un = um;
    um = x;
    x = vn;
    vn = vm;
    vm = x;
    return true;
  };
  if (a.write_c0) {  // C(0), psod.f:89-90 with U2 = U0, V2 = V0
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
      const double u0k = __ldg(a.u0 + k), v0k = __ldg(a.v0 + k);
      q[0] += u0k * u0k;
      q[1] += v0k * v0k;
      q[2] += u0k * v0k;
      q[3] += v0k * u0k;
    }
    if (!reduce_c(q, 0)) return;
  }
  int s0 = 1;
  if (a.start && a.nsteps >= 1) {
    if (!step(0.25 * a.cst, -1, 0)) return;  // psod.f:120-121
    if (!step(0.5 * a.cst, 1, 1)) return;    // psod.f:123-124
    // psod.f:136-141, over the points this CTA's steps write
    auto copy_back = [&](long k) {
      um[k] = __ldg(a.u0 + k);
      vm[k] = (a.copy_quirk && (k & 1)) ? __ldg(a.v0 + k - 1) : __ldg(a.v0 + k);
    };
    if (NDIM == 2 && a.nstrips > 0) {
      const Band B = my_band(a);
      if (B.col < a.nx)
        for (int row = B.r0; row < B.r1; ++row) copy_back((long)row * a.nx + B.col);
    } else {
      for (int k = r.lo + t; k < r.hi; k += kSilThreads) copy_back(k);
    }
    __syncthreads();
    s0 = 2;
  }
  for (int s = s0; s <= a.nsteps; ++s)
    if (!step(a.cst, s, a.slot0 + s)) return;
}

// <u|H u> + <v|H v> and |u|^2 + |v|^2 (EIGENERG, eigenerg.f:56-66): per-CTA
// partials, then one CTA sums them in CTA order
template <int NDIM>
__global__ void __launch_bounds__(kSilThreads) sil_energy_kernel(SilArgs a, double* part,
                                                                 double ef) {
  __shared__ double sp[2], scratch[(kSilThreads / 32) * 8];
  double q[2] = {0.0, 0.0};
  for (long k = (long)blockIdx.x * kSilThreads + threadIdx.x; k < a.n;
       k += (long)gridDim.x * kSilThreads) {
    const double uk = a.u[k], vk = a.v[k];
    int idx[3];
    grid_index<NDIM>(a, (int)k, idx);
    double hu = apply_h_nd<NDIM>(a, a.u, (int)k, 1.0, idx);
    double hv = apply_h_nd<NDIM>(a, a.v, (int)k, 1.0, idx);
    if (a.dm) {  // the potential V - DM EF of a pulse (chpot.f)
      const double de = a.dm[k] * ef;
      hu -= de * uk;
      hv -= de * vk;
    }
    q[0] += uk * hu + vk * hv;
    q[1] += uk * uk + vk * vk;
  }
  block_sum<2>(q, sp, scratch);
  if (threadIdx.x < 2) part[blockIdx.x * 2 + threadIdx.x] = sp[threadIdx.x];
}

__global__ void sum_parts_kernel(const double* part, int nb, double* out) {
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += part[i * 2 + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

// <w_j|u> and <w_j|v> for nvec real vectors w_j (FCORREL of ppsod.f:268-300):
// CTA (x, j) sums a strided slice of the grid for vector j; the per-CTA
// partials are summed in CTA order by project_sum_kernel
constexpr int kProjBlocks = 128;
constexpr int kProjMaxVec = 8;

__global__ void __launch_bounds__(kSilThreads) project_kernel(const double* w, const double* u,
                                                              const double* v, long n,
                                                              double* part) {
  __shared__ double sp[2], scratch[(kSilThreads / 32) * 8];
  const double* wj = w + (size_t)blockIdx.y * n;
  double q[2] = {0.0, 0.0};
  for (long k = (long)blockIdx.x * kSilThreads + threadIdx.x; k < n;
       k += (long)gridDim.x * kSilThreads) {
    const double wk = wj[k];
    q[0] += wk * u[k];
    q[1] += wk * v[k];
  }
  block_sum<2>(q, sp, scratch);
  if (threadIdx.x < 2) part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = sp[threadIdx.x];
}

__global__ void project_sum_kernel(const double* part, int nb, int nvec, double* out) {
  const int t = threadIdx.x;  // 2 per vector
  if (t < 2 * nvec) {
    const int j = t >> 1, c = t & 1;
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += part[((size_t)j * nb + i) * 2 + c];
    out[t] = s;
  }
}

}  // namespace espec

// ---------------------------------------------------------------------------
// grid plan
// ---------------------------------------------------------------------------
using namespace espec;

struct espec_grid_plan {
  int method = ESPEC_SIL, ndim = 1, np[3] = {1, 1, 1};
  long n = 0;
  double shm[3] = {0, 0, 0};
  double dt_fs = 0.0;
  int m = 0, absorb = 0, quirks = 0;
  int precision = ESPEC_FP64;  // ESPEC_MIXED (SIL): FP32 Lanczos vectors and H psi
  int nblocks = 0, nblocks_max = 0;  // CTAs of the cooperative launches (<= co-resident)
  bool loaded = false, has_state = false;
  double *d_vpot = nullptr, *d_mask = nullptr, *d_u = nullptr, *d_v = nullptr;
  double *d_u0 = nullptr, *d_v0 = nullptr, *d_L = nullptr, *d_work = nullptr, *d_wbuf = nullptr;
  double *d_up = nullptr, *d_vp = nullptr;  // PSOD: the state one step back
  double *d_dm = nullptr, *d_ef = nullptr;  // PSOD with a pulse: dipole, field per call
  long n_ef = 0, slot = 0;                  // field entries; steps of the current run
  double *d_part = nullptr, *d_epart = nullptr, *d_eout = nullptr;
  double* d_ppart = nullptr;  // projections: per-CTA partials, then the sums
  unsigned* d_bar = nullptr;
  int* d_err = nullptr;
  double2* d_c = nullptr;
  int c_cap = -1;  // nsteps of the C(t) buffer
};

static void grid_free(espec_grid_plan* p) {
  void* b[] = {p->d_vpot, p->d_mask, p->d_u, p->d_v, p->d_u0, p->d_v0, p->d_L, p->d_work,
               p->d_wbuf, p->d_part, p->d_epart, p->d_eout, p->d_bar, p->d_err, p->d_c,
               p->d_up, p->d_vp, p->d_dm, p->d_ef, p->d_ppart};
  for (void* x : b)
    if (x) cudaFree(x);
}

#define GRID_CK(call)                                        \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_); \
  } while (0)

// Bounded waits of the grid barriers: the poll limit of the next launches
// (espec_set_wait_limit), and the number of next launches whose arrival count
// starts one short (espec_selftest_short_arrivals): their first barrier can
// never complete, so every CTA's wait runs out, sets the error flag and the
// kernel returns -- the time-out path exercised without any fault.
static std::atomic<long> g_wait_limit{kSpinLimit};
static std::atomic<int> g_short_arrivals{0};

// column strips of the PSOD pass on a 2D grid (0: contiguous point ranges):
// used when the CTA count is a multiple of the strip count and every band
// holds at least kBandMinRows rows
static int band_strips(const espec_grid_plan* p) {
  if (p->method != ESPEC_PSOD || p->ndim != 2) return 0;
  const int ns = (p->np[0] + kSilThreads - 1) / kSilThreads;
  if (p->nblocks % ns != 0) return 0;
  const int nb = p->nblocks / ns;
  return p->np[1] / nb >= kBandMinRows ? ns : 0;
}

static SilArgs sil_args(const espec_grid_plan* p) {
  SilArgs a{};
  a.ndim = p->ndim;
  a.nx = p->np[0];
  a.ny = p->np[1];
  a.nz = p->np[2];
  a.n = p->n;
  for (int i = 0; i < 3; ++i) a.shm[i] = i < p->ndim ? p->shm[i] : 0.0;
  // (30 * SHT) with SHT summed over the axes in order (au1d.f, au2di.f)
  double sht = 0.0;
  for (int i = 0; i < p->ndim; ++i) sht += p->shm[i];
  a.sht30 = 30.0 * sht;
  a.inv_nx = 1.0 / p->np[0];
  a.inv_ny = 1.0 / p->np[1];
  a.vpot = p->d_vpot;
  a.mask = p->absorb == ESPEC_ABS_SMOOTHW ? p->d_mask : nullptr;
  a.u = p->d_u;
  a.v = p->d_v;
  a.u0 = p->d_u0;
  a.v0 = p->d_v0;
  a.L = p->d_L;
  a.work = p->d_work;
  a.wbuf = p->d_wbuf;
  a.part = p->d_part;
  a.bar = p->d_bar;
  a.nflag = p->d_bar + 2;
  a.err = p->d_err;
  a.spin_limit = g_wait_limit.load();
  a.c_out = p->d_c;
  a.m = p->m;
  a.quirk = (p->quirks & ESPEC_Q_SIL_INPLACE) != 0;
  a.cst = p->dt_fs / ESPEC_SHFS;
  if (p->method == ESPEC_PSOD) {
    a.cst = 2.0 * p->dt_fs / ESPEC_SHFS;  // psod.f:82
    a.mask = nullptr;
    a.up = p->d_up;
    a.vp = p->d_vp;
    a.vabc = p->d_mask;
    a.kabs = p->absorb == ESPEC_ABS_VOPTIC ? 1 : (p->absorb == ESPEC_ABS_SMOOTHW ? 2 : 0);
    a.copy_quirk = (p->quirks & ESPEC_Q_PSOD_COPY) != 0;
  }
  a.dm = p->d_dm;
  a.ef = p->d_dm ? p->d_ef : nullptr;
  a.nstrips = band_strips(p);
  return a;
}

extern "C" int espec_grid_create(espec_grid_plan** out, int method, int ndim, const int* np,
                                 const double* shm, double dt_fs, int mp, int precision,
                                 int absorb, int quirks) {
  if (!out || !np || !shm) return set_error(ESPEC_EINVAL, "null argument");
  if (method != ESPEC_SIL && method != ESPEC_PSOD)
    return set_error(ESPEC_EINVAL, "grid plans run ESPEC_SIL or ESPEC_PSOD");
  if (precision != ESPEC_FP64 && !(precision == ESPEC_MIXED && method == ESPEC_SIL))
    return set_error(ESPEC_EINVAL, "grid plans run in FP64 (SIL also in ESPEC_MIXED)");
  // the reference-defect form (sil.f:145-148) is not unitary and grows the
  // state, amplifying FP32 rounding: it is kept for the FP64 form, which
  // reproduces the executable's output
  if (precision == ESPEC_MIXED && (quirks & ESPEC_Q_SIL_INPLACE))
    return set_error(ESPEC_EINVAL, "the SIL defect form runs in FP64 only");
  if (ndim < 1 || ndim > 3) return set_error(ESPEC_EINVAL, "ndim must be 1, 2 or 3");
  const bool psod = method == ESPEC_PSOD;
  if (psod) mp = 0;
  if (!psod && (mp < 1 || mp > kSilMaxM))
    return set_error(ESPEC_EINVAL, "Lanczos order must be 1..16");
  if (!psod && absorb == ESPEC_ABS_VOPTIC)
    return set_error(ESPEC_EINVAL, "SIL takes no complex absorbing potential (real Lanczos)");
  if (absorb != ESPEC_ABS_NONE && absorb != ESPEC_ABS_SMOOTHW && absorb != ESPEC_ABS_VOPTIC)
    return set_error(ESPEC_EINVAL, "unknown absorber type");
  if (quirks & ~(psod ? ESPEC_Q_PSOD_COPY : ESPEC_Q_SIL_INPLACE))
    return set_error(ESPEC_EINVAL, "quirk not applicable to this method");
  long n = 1;
  for (int i = 0; i < ndim; ++i) {
    if (np[i] < 1) return set_error(ESPEC_EINVAL, "grid size must be positive");
    n *= np[i];
  }
  if (n > (1L << 30)) return set_error(ESPEC_EINVAL, "grid too large");
  auto* p = new espec_grid_plan;
  p->method = method;
  p->ndim = ndim;
  for (int i = 0; i < ndim; ++i) {
    p->np[i] = np[i];
    p->shm[i] = shm[i];
  }
  p->n = n;
  p->dt_fs = dt_fs;
  p->m = mp;
  p->absorb = absorb;
  p->quirks = quirks;
  p->precision = precision;
  // co-resident CTAs for the cooperative launch
  int dev = 0, nsm = 0, occ = 0;
  const void* kern =
      psod ? (ndim == 1   ? (const void*)psod_kernel<1>
              : ndim == 2 ? (const void*)psod_kernel<2>
                          : (const void*)psod_kernel<3>)
           : (ndim == 1   ? (const void*)sil_kernel<1, false, double>
              : ndim == 2 ? (const void*)sil_kernel<2, false, double>
                          : (const void*)sil_kernel<3, false, double>);
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kSilThreads, 0);
  if (e != cudaSuccess) {
    delete p;
    return set_cuda_error("device query", e);
  }
  long want = (n + kSilThreads - 1) / kSilThreads;
  // one CTA per SM keeps the barriers short; a PSOD pass over a large grid
  // (16 points or more per thread) takes every co-resident CTA instead
  long cap = nsm;
  if (psod && n >= 16L * nsm * kSilThreads) cap = (long)nsm * occ;
  if (cap > (long)nsm * occ) cap = (long)nsm * occ;
  // the fewest CTAs that keep the largest per-CTA share: a grid barrier costs
  // about one arrival per CTA, so 65536 points take 128 CTAs of two 256-point
  // tiles rather than 148 of which some hold one (measured 193 vs 216 us per
  // SIL step of order 12 on 256 x 256)
  if (want > cap) {
    const long per = (want + cap - 1) / cap;
    want = (want + per - 1) / per;
  }
  // a PSOD pass over a large 2D grid runs by column strips: every co-resident
  // CTA, a multiple of the strip count, each band at least kBandMinRows rows
  if (psod && ndim == 2) {
    const long ns = (np[0] + kSilThreads - 1) / kSilThreads, nb = cap / ns;
    if (nb >= 1 && np[1] / nb >= kBandMinRows) want = ns * nb;
  }
  p->nblocks = (int)(want > 0 ? want : 1);
  p->nblocks_max = p->nblocks;
  auto fail = [&](int rc) {
    grid_free(p);
    delete p;
    return rc;
  };
  int rc = 0;
  const size_t nb = (size_t)n * 8;
  double** bufs8[] = {&p->d_vpot, &p->d_mask, &p->d_u, &p->d_v, &p->d_u0, &p->d_v0};
  for (double** b : bufs8)
    if ((rc = ck(cudaMalloc(b, nb), "cudaMalloc"))) return fail(rc);
  if (psod) {
    if ((rc = ck(cudaMalloc(&p->d_up, nb), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_vp, nb), "cudaMalloc"))) return fail(rc);
  } else {
    if ((rc = ck(cudaMalloc(&p->d_L, nb * 2 * mp), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_work, nb * 2), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_wbuf, nb * 2), "cudaMalloc"))) return fail(rc);
  }
  if ((rc = ck(cudaMalloc(&p->d_part, sizeof(double) * 2 * kSilNQ * p->nblocks), "cudaMalloc")))
    return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_epart, sizeof(double) * 2 * 1024), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_eout, sizeof(double) * 2), "cudaMalloc"))) return fail(rc);
  // the 64-bit arrival count, then one handshake flag per CTA
  if ((rc = ck(cudaMalloc(&p->d_bar, sizeof(unsigned) * (2 + p->nblocks_max)), "cudaMalloc")))
    return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_err, sizeof(int)), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMemset(p->d_bar, 0, sizeof(unsigned) * (2 + p->nblocks_max)), "cudaMemset")))
    return fail(rc);
  if ((rc = ck(cudaMemset(p->d_err, 0, sizeof(int)), "cudaMemset"))) return fail(rc);
  *out = p;
  return ESPEC_OK;
}

extern "C" int espec_grid_load(espec_grid_plan* p, const double* vpot, const double* vabc,
                               const double* psi_re, const double* psi_im, int where,
                               void* stream) {
  if (!p || !vpot || !psi_re) return set_error(ESPEC_EINVAL, "null argument");
  if (p->absorb != ESPEC_ABS_NONE && !vabc) return set_error(ESPEC_EINVAL, "absorber table missing");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const size_t nb = (size_t)p->n * 8;
  GRID_CK(cudaMemcpyAsync(p->d_vpot, vpot, nb, kind, st));
  if (p->absorb != ESPEC_ABS_NONE) GRID_CK(cudaMemcpyAsync(p->d_mask, vabc, nb, kind, st));
  GRID_CK(cudaMemcpyAsync(p->d_u0, psi_re, nb, kind, st));
  if (psi_im) {
    GRID_CK(cudaMemcpyAsync(p->d_v0, psi_im, nb, kind, st));
  } else {
    GRID_CK(cudaMemsetAsync(p->d_v0, 0, nb, st));
  }
  GRID_CK(cudaMemcpyAsync(p->d_u, p->d_u0, nb, cudaMemcpyDeviceToDevice, st));
  GRID_CK(cudaMemcpyAsync(p->d_v, p->d_v0, nb, cudaMemcpyDeviceToDevice, st));
  p->loaded = true;
  p->has_state = false;
  return ESPEC_OK;
}

static int grid_launch(espec_grid_plan* p, int nsteps, bool from_start, cudaStream_t st) {
  if (p->c_cap != nsteps) {
    if (p->d_c) cudaFree(p->d_c);
    p->d_c = nullptr;
    GRID_CK(cudaMalloc(&p->d_c, sizeof(double2) * ((size_t)nsteps + 1)));
    p->c_cap = nsteps;
  }
  const size_t nb = (size_t)p->n * 8;
  if (from_start) {
    GRID_CK(cudaMemcpyAsync(p->d_u, p->d_u0, nb, cudaMemcpyDeviceToDevice, st));
    GRID_CK(cudaMemcpyAsync(p->d_v, p->d_v0, nb, cudaMemcpyDeviceToDevice, st));
  }
  // the 64-bit arrival count starts at 0, or at 2^64 - 1 (one short of the
  // first barrier's G arrivals, modulo 2^64) for a self-test launch
  const bool short_start = g_short_arrivals.load() > 0 && g_short_arrivals.fetch_sub(1) > 0;
  GRID_CK(cudaMemsetAsync(p->d_bar, short_start ? 0xFF : 0, sizeof(unsigned) * 2, st));
  GRID_CK(cudaMemsetAsync(p->d_bar + 2, 0, sizeof(unsigned) * p->nblocks, st));
  GRID_CK(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
  SilArgs a = sil_args(p);
  a.nsteps = nsteps;
  a.write_c0 = from_start ? 1 : 0;
  if (p->method == ESPEC_PSOD) {
    if (from_start) {  // psod.f:83-88: U2 = U1 = U0, V2 = V1 = V0
      GRID_CK(cudaMemcpyAsync(p->d_up, p->d_u0, nb, cudaMemcpyDeviceToDevice, st));
      GRID_CK(cudaMemcpyAsync(p->d_vp, p->d_v0, nb, cudaMemcpyDeviceToDevice, st));
    } else if (!p->has_state) {
      return set_error(ESPEC_EINVAL, "a PSOD plan continues a run: call espec_grid_run first");
    }
    a.start = from_start ? 1 : 0;
    a.slot0 = from_start ? 0 : p->slot;
    if (p->d_dm && a.slot0 + nsteps >= p->n_ef)
      return set_error(ESPEC_EINVAL, "the pulse field table ends before the run does");
    void* args[] = {&a};
    const void* kern = p->ndim == 1   ? (const void*)psod_kernel<1>
                       : p->ndim == 2 ? (const void*)psod_kernel<2>
                                      : (const void*)psod_kernel<3>;
    GRID_CK(cudaLaunchCooperativeKernel(kern, dim3(p->nblocks),
                                        dim3(kSilThreads), args, 0, st));
    // the kernel swaps the roles of the two state buffers once per step
    const long swaps = from_start ? (nsteps >= 1 ? nsteps + 1 : 0) : nsteps;
    if (swaps & 1) {
      std::swap(p->d_u, p->d_up);
      std::swap(p->d_v, p->d_vp);
    }
    p->has_state = true;
    p->slot = a.slot0 + nsteps;
    return ESPEC_OK;
  }
  a.slot0 = from_start ? 0 : p->slot;
  if (p->d_dm && a.slot0 + nsteps >= p->n_ef)
    return set_error(ESPEC_EINVAL, "the pulse field table ends before the run does");
  void* args[] = {&a};
  // the CTAs' own Lanczos vectors in shared memory when they fit
  const long chunk = (p->n + p->nblocks - 1) / p->nblocks;
  const bool mixed = p->precision == ESPEC_MIXED;
  const size_t dyn = sil_vec_smem(p->m, chunk, mixed ? 4 : 8);
  const void* ks = mixed ? (p->ndim == 1   ? (const void*)sil_kernel<1, true, float>
                            : p->ndim == 2 ? (const void*)sil_kernel<2, true, float>
                                           : (const void*)sil_kernel<3, true, float>)
                         : (p->ndim == 1   ? (const void*)sil_kernel<1, true, double>
                            : p->ndim == 2 ? (const void*)sil_kernel<2, true, double>
                                           : (const void*)sil_kernel<3, true, double>);
  const void* kg = mixed ? (p->ndim == 1   ? (const void*)sil_kernel<1, false, float>
                            : p->ndim == 2 ? (const void*)sil_kernel<2, false, float>
                                           : (const void*)sil_kernel<3, false, float>)
                         : (p->ndim == 1   ? (const void*)sil_kernel<1, false, double>
                            : p->ndim == 2 ? (const void*)sil_kernel<2, false, double>
                                           : (const void*)sil_kernel<3, false, double>);
  int dev = 0, optin = 0;
  cudaFuncAttributes fa{};
  GRID_CK(cudaGetDevice(&dev));
  GRID_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  GRID_CK(cudaFuncGetAttributes(&fa, ks));
  const bool in_smem = fa.sharedSizeBytes + dyn <= (size_t)optin;
  if (in_smem)
    GRID_CK(cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  GRID_CK(cudaLaunchCooperativeKernel(in_smem ? ks : kg, dim3(p->nblocks), dim3(kSilThreads),
                                      args, in_smem ? dyn : 0, st));
  p->slot = a.slot0 + nsteps;
  return ESPEC_OK;
}

extern "C" int espec_grid_run(espec_grid_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_grid_load has not been called");
  return grid_launch(p, nsteps, true, (cudaStream_t)stream);
}

extern "C" int espec_grid_continue(espec_grid_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_grid_load has not been called");
  return grid_launch(p, nsteps, false, (cudaStream_t)stream);
}

extern "C" int espec_grid_results(espec_grid_plan* p, double* c_re, double* c_im, double* psi_re,
                                  double* psi_im, int where, void* stream) {
  if (!p || p->c_cap < 0) return set_error(ESPEC_EINVAL, "no results: run the plan first");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const size_t nc = (size_t)p->c_cap + 1;
  if (c_re) GRID_CK(cudaMemcpy2DAsync(c_re, 8, p->d_c, 16, 8, nc, kind, st));
  if (c_im) GRID_CK(cudaMemcpy2DAsync(c_im, 8, (char*)p->d_c + 8, 16, 8, nc, kind, st));
  const size_t nb = (size_t)p->n * 8;
  if (psi_re) GRID_CK(cudaMemcpyAsync(psi_re, p->d_u, nb, kind, st));
  if (psi_im) GRID_CK(cudaMemcpyAsync(psi_im, p->d_v, nb, kind, st));
  int err = 0;
  GRID_CK(cudaMemcpyAsync(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  GRID_CK(cudaStreamSynchronize(st));
  if (err) return set_error(ESPEC_ECUDA, "a grid barrier of the SIL kernel timed out");
  return ESPEC_OK;
}

extern "C" int espec_grid_energies_at(espec_grid_plan* p, double ef, double* e, double* norm,
                                      void* stream) {
  if (!p || !e || !norm) return set_error(ESPEC_EINVAL, "null argument");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_grid_load has not been called");
  cudaStream_t st = (cudaStream_t)stream;
  SilArgs a = sil_args(p);
  long nbk = (p->n + kSilThreads - 1) / kSilThreads;
  if (nbk > 1024) nbk = 1024;
  if (p->ndim == 1) sil_energy_kernel<1><<<(int)nbk, kSilThreads, 0, st>>>(a, p->d_epart, ef);
  else if (p->ndim == 2) sil_energy_kernel<2><<<(int)nbk, kSilThreads, 0, st>>>(a, p->d_epart, ef);
  else sil_energy_kernel<3><<<(int)nbk, kSilThreads, 0, st>>>(a, p->d_epart, ef);
  GRID_CK(cudaGetLastError());
  sum_parts_kernel<<<1, 32, 0, st>>>(p->d_epart, (int)nbk, p->d_eout);
  GRID_CK(cudaGetLastError());
  double h[2];
  GRID_CK(cudaMemcpyAsync(h, p->d_eout, sizeof h, cudaMemcpyDeviceToHost, st));
  GRID_CK(cudaStreamSynchronize(st));
  *e = h[0];
  *norm = h[1];
  return ESPEC_OK;
}

extern "C" int espec_grid_previous(espec_grid_plan* p, double* psi_re, double* psi_im, int where,
                                   void* stream) {
  if (!p || p->method != ESPEC_PSOD || !p->has_state)
    return set_error(ESPEC_EINVAL, "previous state exists for run PSOD plans only");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const size_t nb = (size_t)p->n * 8;
  if (psi_re) GRID_CK(cudaMemcpyAsync(psi_re, p->d_up, nb, kind, st));
  if (psi_im) GRID_CK(cudaMemcpyAsync(psi_im, p->d_vp, nb, kind, st));
  int err = 0;
  GRID_CK(cudaMemcpyAsync(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  GRID_CK(cudaStreamSynchronize(st));
  if (err) return set_error(ESPEC_ECUDA, "a grid barrier of the PSOD kernel timed out");
  return ESPEC_OK;
}

extern "C" int espec_grid_energies(espec_grid_plan* p, double* e, double* norm, void* stream) {
  return espec_grid_energies_at(p, 0.0, e, norm, stream);
}

extern "C" int espec_grid_set_pulse(espec_grid_plan* p, const double* dm, const double* ef,
                                    long ncalls, int where) {
  if (!p) return set_error(ESPEC_EINVAL, "null plan");
  if (!dm || !ef || ncalls < 1) return set_error(ESPEC_EINVAL, "dipole and field table needed");
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (p->d_ef) cudaFree(p->d_ef);
  p->d_ef = nullptr;
  p->n_ef = 0;
  if (!p->d_dm) GRID_CK(cudaMalloc(&p->d_dm, (size_t)p->n * 8));
  GRID_CK(cudaMalloc(&p->d_ef, (size_t)ncalls * 8));
  GRID_CK(cudaMemcpy(p->d_dm, dm, (size_t)p->n * 8, kind));
  GRID_CK(cudaMemcpy(p->d_ef, ef, (size_t)ncalls * 8, kind));
  p->n_ef = ncalls;
  return ESPEC_OK;
}

extern "C" int espec_grid_project(espec_grid_plan* p, const double* w, int nvec, double* out,
                                  void* stream) {
  if (!p || !w || !out) return set_error(ESPEC_EINVAL, "null argument");
  if (nvec < 1 || nvec > kProjMaxVec) return set_error(ESPEC_EINVAL, "1..8 projection vectors");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_grid_load has not been called");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nsum = (size_t)kProjMaxVec * kProjBlocks * 2;
  if (!p->d_ppart) GRID_CK(cudaMalloc(&p->d_ppart, sizeof(double) * (nsum + 2 * kProjMaxVec)));
  long nb = (p->n + kSilThreads - 1) / kSilThreads;
  if (nb > kProjBlocks) nb = kProjBlocks;
  project_kernel<<<dim3((unsigned)nb, (unsigned)nvec), kSilThreads, 0, st>>>(w, p->d_u, p->d_v, p->n,
                                                                             p->d_ppart);
  GRID_CK(cudaGetLastError());
  project_sum_kernel<<<1, 2 * kProjMaxVec, 0, st>>>(p->d_ppart, (int)nb, nvec, p->d_ppart + nsum);
  GRID_CK(cudaGetLastError());
  GRID_CK(cudaMemcpyAsync(out, p->d_ppart + nsum, sizeof(double) * 2 * nvec,
                          cudaMemcpyDeviceToHost, st));
  GRID_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}

extern "C" int espec_set_wait_limit(long polls) {
  if (polls < 0) return set_error(ESPEC_EINVAL, "negative poll limit");
  g_wait_limit.store(polls == 0 ? kSpinLimit : polls);
  return ESPEC_OK;
}

extern "C" int espec_selftest_short_arrivals(int launches) {
  if (launches < 0) return set_error(ESPEC_EINVAL, "negative launch count");
  g_short_arrivals.store(launches);
  return ESPEC_OK;
}

extern "C" int espec_grid_set_ctas(espec_grid_plan* p, int nctas) {
  if (!p || nctas < 0) return set_error(ESPEC_EINVAL, "null plan or negative CTA count");
  if (nctas > p->nblocks_max)
    return set_error(ESPEC_EINVAL, "more CTAs than the plan's co-resident maximum");
  p->nblocks = nctas == 0 ? p->nblocks_max : nctas;
  return ESPEC_OK;
}

extern "C" long espec_grid_npoints(const espec_grid_plan* p) { return p ? p->n : -1; }

extern "C" void espec_grid_destroy(espec_grid_plan* p) {
  if (!p) return;
  grid_free(p);
  delete p;
}

extern "C" int espec_grid_basis(espec_grid_plan* p, int chain, double* dst, int ld, int where,
                                void* stream) {
  if (!p || !dst || chain < 0 || chain > 1) return set_error(ESPEC_EINVAL, "bad argument");
  if (p->c_cap < 0) return set_error(ESPEC_EINVAL, "no basis: run the plan first");
  if (ld < p->n) return set_error(ESPEC_EINVAL, "leading dimension below the grid size");
  if (p->precision != ESPEC_FP64)
    return set_error(ESPEC_EINVAL, "a mixed plan keeps its Lanczos basis in FP32");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const double* src = p->d_L + (size_t)chain * p->m * p->n;
  GRID_CK(cudaMemcpy2DAsync(dst, (size_t)ld * 8, src, (size_t)p->n * 8, (size_t)p->n * 8, p->m,
                            kind, st));
  if (where == ESPEC_MEM_HOST) GRID_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}
