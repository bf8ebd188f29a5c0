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
__device__ bool grid_reduce(const SilArgs& a, const double* sp, double* st, int nq,
                            int* s_flag, double* s_red /* kSilThreads doubles */,
                            unsigned& phase) {
  const int b = blockIdx.x, G = gridDim.x, t = threadIdx.x;
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
  // to 16 loads in flight, then the R partial sums in order
  double* red = s_red;
  const int R = nq > 0 ? min(kSilThreads / nq, 32) : 1;
  if (t < R * nq) {
    const int q = t % nq, r = t / nq;
    double acc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] = 0.0;
    for (int i0 = r; i0 < G; i0 += 16 * R) {
      double x[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int i = i0 + j * R;
        x[j] = i < G ? __ldcg(part + (long)i * kSilNQ + q) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] += x[j];
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 16; ++j) s += acc[j];
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
template <int NDIM>
__device__ __forceinline__ double apply_h_nd(const SilArgs& a, const double* x, int k, double d,
                                             const int (&idx)[3]) {
  const int len[3] = {a.nx, a.ny, a.nz}, str[3] = {1, a.nx, a.nx * a.ny};
  double xm2[NDIM], xm1[NDIM], xp1[NDIM], xp2[NDIM];
#pragma unroll
  for (int ax = 0; ax < NDIM; ++ax) {
    const int i = idx[ax], st = str[ax], L = len[ax];
    xm2[ax] = ld_state(x + (i >= 2 ? k - 2 * st : k));
    xm1[ax] = ld_state(x + (i >= 1 ? k - st : k));
    xp1[ax] = ld_state(x + (i + 1 < L ? k + st : k));
    xp2[ax] = ld_state(x + (i + 2 < L ? k + 2 * st : k));
  }
  double s = (a.sht30 + __ldg(a.vpot + k)) * (ld_state(x + k) * d);
#pragma unroll
  for (int ax = 0; ax < NDIM; ++ax) {
    const double h = a.shm[ax];
    const int i = idx[ax], L = len[ax];
    if (i >= 2) s += h * (xm2[ax] * d);
    if (i >= 1) s += -16.0 * h * (xm1[ax] * d);
    if (i + 1 < L) s += -16.0 * h * (xp1[ax] * d);
    if (i + 2 < L) s += h * (xp2[ax] * d);
  }
  return s;
}

// Krylov coefficients of both chains (every CTA computes the same values):
// Z = exp(-i cst T) by Taylor series (degree kTaylor) of T scaled to norm
// <= 1/2, then squared back.  out[0] = Re Z y_u, out[1] = Im Z y_u (or
// Im(Z^2) y_u / 2 in the reference-defect form), out[2] = Re Z y_v,
// out[3] = -Im Z y_v.
constexpr int kTaylor = 14;  // |B| <= 1/2: truncation 0.5^15/15! = 2.3e-17
constexpr int kMM = kSilMaxM * kSilMaxM;

struct KrylovSmem {
  double2 X[2][2][kMM];  // [buffer][chain], ping-pong
};

__device__ void krylov_coeffs(int m, double cst, int quirk, const double (*al)[kSilMaxM],
                              const double (*bt)[kSilMaxM], const double (*y)[kSilMaxM],
                              const int* active, KrylovSmem& ks, double (*out)[kSilMaxM]) {
  __shared__ int s_sq[2];
  __shared__ double s_scale[2];
  const int t = threadIdx.x;
  if (t < 2) {
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) {
      double r = fabs(al[t][i]);
      if (i > 0) r += fabs(bt[t][i - 1]);
      if (i + 1 < m) r += fabs(bt[t][i]);
      nrm = fmax(nrm, r);
    }
    nrm *= fabs(cst);
    int sq = 0;
    while (nrm > 0.5 && sq < 60) {
      nrm *= 0.5;
      ++sq;
    }
    s_sq[t] = sq;
    s_scale[t] = ldexp(cst, -sq);
  }
  // buffer 0 = I
  for (int e = t; e < 2 * kMM; e += blockDim.x) {
    const int c = e / kMM, i = (e % kMM) / kSilMaxM, j = e % kSilMaxM;
    ks.X[0][c][i * kSilMaxM + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  // Horner: P <- I + B P / k, B = -i scale T (T tridiagonal)
  int cur = 0;
  for (int k = kTaylor; k >= 1; --k) {
    const double rk = 1.0 / k;
    for (int e = t; e < 2 * kMM; e += blockDim.x) {
      const int c = e / kMM, i = (e % kMM) / kSilMaxM, j = e % kSilMaxM;
      if (i >= m || j >= m) continue;
      const double2* P = ks.X[cur][c];
      const double sc = s_scale[c];
      // (B P)_{ij} = sum_l (-i sc T_il) P_lj = sum_l sc T_il (Im P_lj, -Re P_lj)
      const double tii = sc * al[c][i];
      const double2 pii = P[i * kSilMaxM + j];
      double re = tii * pii.y, im = -tii * pii.x;
      if (i > 0) {
        const double tl = sc * bt[c][i - 1];
        const double2 q = P[(i - 1) * kSilMaxM + j];
        re += tl * q.y;
        im -= tl * q.x;
      }
      if (i + 1 < m) {
        const double tu = sc * bt[c][i];
        const double2 q = P[(i + 1) * kSilMaxM + j];
        re += tu * q.y;
        im -= tu * q.x;
      }
      ks.X[cur ^ 1][c][i * kSilMaxM + j] = make_double2((i == j ? 1.0 : 0.0) + re * rk, im * rk);
    }
    __syncthreads();
    cur ^= 1;
  }
  // squaring back; the defect form also needs Z^2 of chain 0
  int cc[2] = {cur, cur};
  const int nsq = max(s_sq[0], s_sq[1]) + (quirk ? 1 : 0);
  for (int q = 0; q < nsq; ++q) {
    for (int e = t; e < 2 * kMM; e += blockDim.x) {
      const int c = e / kMM, i = (e % kMM) / kSilMaxM, j = e % kSilMaxM;
      if (i >= m || j >= m) continue;
      if (q > s_sq[c] || (q == s_sq[c] && !(quirk && c == 0))) continue;
      const double2* P = ks.X[cc[c]][c];
      double re = 0.0, im = 0.0;
      for (int l = 0; l < m; ++l) {
        const double2 x = P[i * kSilMaxM + l], z = P[l * kSilMaxM + j];
        re += x.x * z.x - x.y * z.y;
        im += x.x * z.y + x.y * z.x;
      }
      ks.X[cc[c] ^ 1][c][i * kSilMaxM + j] = make_double2(re, im);
    }
    __syncthreads();
    for (int c = 0; c < 2; ++c)
      if (q < s_sq[c]) cc[c] ^= 1;
  }
  // coefficients: Z = X[cc[c]][c]; Z^2 of chain 0 in the other buffer
  if (t < 2 * kSilMaxM) {
    const int c = t / kSilMaxM, i = t % kSilMaxM;
    if (i < m) {
      const double2* Z = ks.X[cc[c]][c];
      const double2* Z2 = ks.X[cc[0] ^ 1][0];
      double re = 0.0, im = 0.0, im2 = 0.0;
      if (active[c]) {
        for (int j = 0; j < m; ++j) {
          const double2 z = Z[i * kSilMaxM + j];
          re += z.x * y[c][j];
          im += z.y * y[c][j];
          if (quirk && c == 0) im2 += Z2[i * kSilMaxM + j].y * y[c][j];
        }
      }
      if (c == 0) {
        out[0][i] = re;
        out[1][i] = quirk ? 0.5 * im2 : im;
      } else {
        out[2][i] = re;
        out[3][i] = -im;
      }
    }
  }
  __syncthreads();
}

}  // namespace

// per-chain slots of the dot products of one Lanczos iteration:
// [al_raw, proj, g_it, d_0..d_{it-1}, g_0..g_{it-1}]
__device__ __forceinline__ int slot_of(int c, int it, int i) { return c * (3 + 2 * it) + i; }

// warp sums of acc[0..3+2it) into ws[warp][slot]
__device__ __forceinline__ void warp_sums(const double (&acc)[3 + 2 * kSilMaxM], int c, int it,
                                          double* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 3 + 2 * kSilMaxM; ++i) {
    const bool valid = i < 3 || (i < 3 + kSilMaxM ? i - 3 < it : i - 3 - kSilMaxM < it);
    if (!valid) continue;  // uniform over the CTA
    double s = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const int slot = i < 3 ? i : (i < 3 + kSilMaxM ? i : i - kSilMaxM + it);
    if (lane == 0) ws[warp * kSilNQ + slot_of(c, it, slot)] = s;
  }
}

template <int NDIM>
__global__ void __launch_bounds__(kSilThreads, 1) sil_kernel(SilArgs a) {
  __shared__ double sp[kSilNQ], st[kSilNQ], scratch[(kSilThreads / 32) * 8];
  __shared__ double ws[(kSilThreads / 32) * kSilNQ];
  __shared__ double s_red[kSilThreads];
  __shared__ int s_flag[2];
  __shared__ double s_al[2][kSilMaxM], s_bt[2][kSilMaxM], s_proj[2][kSilMaxM];
  __shared__ double s_r[2][kSilMaxM], s_coef[4][kSilMaxM];
  __shared__ double s_bt0[2];
  __shared__ int s_active[2];
  __shared__ KrylovSmem ks;
  const Range r = my_range(a.n);
  const int t = threadIdx.x;
  const long n = a.n;
  const int m = a.m;
  unsigned phase = 0;  // grid barriers passed in this launch
  constexpr int NW = kSilThreads / 32;

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
      if (!grid_reduce(a, sp, st, 6, s_flag, s_red, phase)) return;
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
    // ---- m Lanczos iterations of both chains
    for (int it = 0; it < m; ++it) {
      // vi = work/bt0, w = H vi - bt0 v_prev at the CTA's points, and the dot
      // products of the iteration accumulated per thread
      for (int c = 0; c < 2; ++c) {
        const double bt0 = s_bt0[c];
        // vi = work * (1/bt0) here and for the stencil's neighbours alike, so
        // the stencil sees exactly the stored vi
        const double rb = 1.0 / bt0;
        const bool act = s_active[c];
        const double* x = c ? a.v : a.u;
        const double* src = it == 0 ? x : a.work + c * n;
        double* Lc = a.L + (long)c * m * n;
        double acc[3 + 2 * kSilMaxM];
#pragma unroll
        for (int i = 0; i < 3 + 2 * kSilMaxM; ++i) acc[i] = 0.0;
        if (act) {
          // vi and w at point k, the iteration's dot products accumulated
          auto point = [&](int k, double& vi_out, double& w_out) __attribute__((always_inline)) {
            double lq[kSilMaxM];
#pragma unroll
            for (int q = 0; q < kSilMaxM; ++q) lq[q] = q < it ? ld_state(Lc + (long)q * n + k) : 0.0;
            const double vi = ld_state(src + k) * rb;
            const double vprev = it ? ld_state(Lc + (long)(it - 1) * n + k) : 0.0;
            int idx[3];
            grid_index<NDIM>(a, k, idx);
            double hv = apply_h_nd<NDIM>(a, src, k, rb, idx);
            if (a.dm) hv -= __ldg(a.dm + k) * efs * vi;
            const double w = hv - bt0 * vprev;
            const double xk = ld_state(x + k);
            vi_out = vi;
            w_out = w;
            acc[0] += vi * w;
            acc[1] += vi * xk;
            acc[2] += vi * vi;
#pragma unroll
            for (int q = 0; q < kSilMaxM; ++q) {
              acc[3 + q] += w * lq[q];
              acc[3 + kSilMaxM + q] += vi * lq[q];
            }
          };
          // two points per thread at a time with no branch between them and
          // the stores after both, so their loads are in flight together
          int k0 = r.lo + t;
          for (; k0 + kSilThreads < r.hi; k0 += 2 * kSilThreads) {
            double vi0, w0, vi1, w1;
            point(k0, vi0, w0);
            point(k0 + kSilThreads, vi1, w1);
            Lc[(long)it * n + k0] = vi0;
            a.wbuf[c * n + k0] = w0;
            Lc[(long)it * n + k0 + kSilThreads] = vi1;
            a.wbuf[c * n + k0 + kSilThreads] = w1;
          }
          for (; k0 < r.hi; k0 += kSilThreads) {
            double vi0, w0;
            point(k0, vi0, w0);
            Lc[(long)it * n + k0] = vi0;
            a.wbuf[c * n + k0] = w0;
          }
        } else {
          for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
            Lc[(long)it * n + k] = 0.0;
            a.wbuf[c * n + k] = 0.0;
          }
        }
        warp_sums(acc, c, it, ws);
      }
      __syncthreads();
      const int nq = 2 * (3 + 2 * it);
      for (int q = t; q < nq; q += kSilThreads) {
        double sum = 0.0;
        for (int w = 0; w < NW; ++w) sum += ws[w * kSilNQ + q];
        sp[q] = sum;
      }
      __syncthreads();
      if (!grid_reduce(a, sp, st, nq, s_flag, s_red, phase)) return;
      if (t < 2) {
        const int c = t, b0 = slot_of(c, it, 0);
        const double al = st[b0];
        s_al[c][it] = al;
        s_proj[c][it] = st[b0 + 1];
        // reort.f against the it+1 stored vectors: r_q = <w - al vi, L_q>
        for (int q = 0; q < it; ++q) s_r[c][q] = st[b0 + 3 + q] - al * st[b0 + 3 + it + q];
        s_r[c][it] = al - al * st[b0 + 2];
      }
      __syncthreads();
      if (it == m - 1) break;  // the last residual is not needed (BT(M) unused)
      // both chains at each point: their loads are in flight together
      double nn[2] = {0.0, 0.0};
      for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
        double res[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const double al = s_al[c][it];
          const double* Lc = a.L + (long)c * m * n;
          double lq[kSilMaxM + 1];
#pragma unroll
          for (int q = 0; q <= kSilMaxM; ++q) lq[q] = q <= it ? ld_state(Lc + (long)q * n + k) : 0.0;
          double acc = ld_state(a.wbuf + c * n + k);
          double vi = 0.0;
#pragma unroll
          for (int q = 0; q <= kSilMaxM; ++q)
            if (q == it) vi = lq[q];
          acc -= al * vi;
#pragma unroll
          for (int q = 0; q <= kSilMaxM; ++q)
            if (q <= it) acc -= s_r[c][q] * lq[q];
          res[c] = acc;
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          a.work[c * n + k] = res[c];
          nn[c] += res[c] * res[c];
        }
      }
      block_sum<2>(nn, sp, scratch);
      if (!grid_reduce(a, sp, st, 2, s_flag, s_red, phase)) return;
      if (t < 2) {
        s_bt[t][it] = sqrt(st[t]);
        s_bt0[t] = s_bt[t][it];
      }
      __syncthreads();
    }
    // ---- Krylov exponential and the new state
    krylov_coeffs(m, a.cst, a.quirk, s_al, s_bt, s_proj, s_active, ks, s_coef);
    const double* Lu = a.L;
    const double* Lv = a.L + (long)m * n;
#pragma unroll
    for (int i = 0; i < 6; ++i) qn[i] = 0.0;
    for (int k = r.lo + t; k < r.hi; k += kSilThreads) {
      double lu[kSilMaxM], lv[kSilMaxM];
#pragma unroll
      for (int j = 0; j < kSilMaxM; ++j) {
        lu[j] = j < m ? ld_state(Lu + (long)j * n + k) : 0.0;
        lv[j] = j < m ? ld_state(Lv + (long)j * n + k) : 0.0;
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

template <int NDIM>
__device__ __forceinline__ void psod_dispatch(const SilArgs& a, Range r, const double* un,
                                              const double* vn, double* um, double* vm, double c,
                                              double e, double (&q)[4]) {
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
    for (int k = r.lo + t; k < r.hi; k += kSilThreads) {  // psod.f:136-141
      um[k] = __ldg(a.u0 + k);
      vm[k] = (a.copy_quirk && (k & 1)) ? __ldg(a.v0 + k - 1) : __ldg(a.v0 + k);
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
  return a;
}

extern "C" int espec_grid_create(espec_grid_plan** out, int method, int ndim, const int* np,
                                 const double* shm, double dt_fs, int mp, int precision,
                                 int absorb, int quirks) {
  if (!out || !np || !shm) return set_error(ESPEC_EINVAL, "null argument");
  if (method != ESPEC_SIL && method != ESPEC_PSOD)
    return set_error(ESPEC_EINVAL, "grid plans run ESPEC_SIL or ESPEC_PSOD");
  if (precision != ESPEC_FP64) return set_error(ESPEC_EINVAL, "grid plans run in FP64");
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
  // co-resident CTAs for the cooperative launch
  int dev = 0, nsm = 0, occ = 0;
  const void* kern =
      psod ? (ndim == 1   ? (const void*)psod_kernel<1>
              : ndim == 2 ? (const void*)psod_kernel<2>
                          : (const void*)psod_kernel<3>)
           : (ndim == 1   ? (const void*)sil_kernel<1>
              : ndim == 2 ? (const void*)sil_kernel<2>
                          : (const void*)sil_kernel<3>);
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
  if ((rc = ck(cudaMalloc(&p->d_bar, sizeof(unsigned) * 2), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_err, sizeof(int)), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMemset(p->d_bar, 0, sizeof(unsigned) * 2), "cudaMemset"))) return fail(rc);
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
  const void* kern = p->ndim == 1   ? (const void*)sil_kernel<1>
                     : p->ndim == 2 ? (const void*)sil_kernel<2>
                                    : (const void*)sil_kernel<3>;
  GRID_CK(cudaLaunchCooperativeKernel(kern, dim3(p->nblocks), dim3(kSilThreads),
                                      args, 0, st));
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
  cudaStream_t st = (cudaStream_t)stream;
  const cudaMemcpyKind kind =
      where == ESPEC_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const double* src = p->d_L + (size_t)chain * p->m * p->n;
  GRID_CK(cudaMemcpy2DAsync(dst, (size_t)ld * 8, src, (size_t)p->n * 8, (size_t)p->n * 8, p->m,
                            kind, st));
  if (where == ESPEC_MEM_HOST) GRID_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}
