// eig.cu -- batched initial-state eigensolver on 2D grids (eSPec's LANCZSG,
// lanczsc.f:56-120, with LNZ lnz.f:76-119 and REORT reort.f:65-80), FP64.
//
// One CTA per problem (one potential): for each of nstates target states,
// explicitly restarted Lanczos -- m Lanczos steps with full classical
// Gram-Schmidt reorthogonalisation from the current vector, the lowest Ritz
// pair of the m x m tridiagonal matrix, restart from that Ritz vector --
// until the true residual |H v - theta v| (one more H*v) is at most tol.  The
// states already found are locked: projected out of every restart vector and
// kept in the reorthogonalisation set (without that, the reference's K-th
// Ritz vector can settle on a higher state; espec.f:896-903 restricts
// LANCZSG to the ground state).
// DSTEVX('V','I') is replaced by multisection on the Sturm count (one warp,
// 33 points per round) and inverse iteration for the Ritz vector.  Every
// application of H is counted: the count is the cost metric of the solver.
// Cold start: the reference's LCG vectors (rans.f:38-39, NSEED = 1, first N
// draws discarded, lanczsc.f:56-62); warm start: any given vectors.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {
namespace {

constexpr int kEigThreads = 1024;  // 32 warps: enough loads in flight per SM
constexpr int kEigMaxM = 40;      // NREORT = 40 in lanczsc.f:55
constexpr int kEigMaxStates = 16;  // locked states held in the reorthogonalisation

struct EigArgs {
  int nx, ny, n;
  double shm[2], sht30;
  const double* vpot;   // [nprob][n]
  const double* start;  // [nprob][nstates][n]
  double* L;            // [nprob][m][n]
  double* work;         // [nprob][n]
  double* vec;          // [nprob][nstates][n]
  double* eval;         // [nprob][nstates]
  double* resid;        // [nprob][nstates]
  int* matvecs;         // [nprob][nstates]
  int nstates, m, maxrest;
  double tol;
};

// H_FD x (au2di.f:57-225) at point k of an nx x ny grid, x scaled by d
__device__ __forceinline__ double hx(const EigArgs& a, const double* V, const double* x, int k,
                                     double d) {
  const int i = k % a.nx, j = k / a.nx;
  double s = (a.sht30 + V[k]) * (x[k] * d);
  const double h0 = a.shm[0], h1 = a.shm[1];
  if (i >= 2) s += h0 * (x[k - 2] * d);
  if (i >= 1) s += -16.0 * h0 * (x[k - 1] * d);
  if (i + 1 < a.nx) s += -16.0 * h0 * (x[k + 1] * d);
  if (i + 2 < a.nx) s += h0 * (x[k + 2] * d);
  const int sy = a.nx;
  if (j >= 2) s += h1 * (x[k - 2 * sy] * d);
  if (j >= 1) s += -16.0 * h1 * (x[k - sy] * d);
  if (j + 1 < a.ny) s += -16.0 * h1 * (x[k + sy] * d);
  if (j + 2 < a.ny) s += h1 * (x[k + 2 * sy] * d);
  return s;
}

// CTA sum of cnt per-thread values (acc[0..cnt)) into out[0..cnt)
template <int MAXV>
__device__ __forceinline__ void cta_sums(const double (&acc)[MAXV], int cnt, double* ws,
                                         double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < MAXV; ++i) {
    if (i >= cnt) break;
    double s = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) ws[warp * MAXV + i] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kEigThreads / 32; ++w) s += ws[w * MAXV + i];
    out[i] = s;
  }
  __syncthreads();
}

// as cta_sums for the slots [0, e1) and [b2, e2) of acc only
template <int MAXV>
__device__ __forceinline__ void cta_sums2(const double (&acc)[MAXV], int e1, int b2, int e2,
                                          double* ws, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < MAXV; ++i) {
    if (!(i < e1 || (i >= b2 && i < e2))) continue;  // uniform over the CTA
    double s = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) ws[warp * MAXV + i] = s;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < MAXV; i += blockDim.x) {
    if (!(i < e1 || (i >= b2 && i < e2))) continue;
    double s = 0.0;
    for (int w = 0; w < kEigThreads / 32; ++w) s += ws[w * MAXV + i];
    out[i] = s;
  }
  __syncthreads();
}

// red[q] = <x, Y_q>, q < nl + nlock, with Y_q = L_q (q < nl) or lock_(q-nl):
// one warp per vector, lanes striding the points (coalesced streams, one per
// warp); x is read from L1/L2 by every warp
__device__ __forceinline__ void warp_dots(const double* x, const double* L, int nl,
                                          const double* lock, int nlock, int n, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = warp; q < nl + nlock; q += kEigThreads / 32) {
    const double* y = q < nl ? L + (long)q * n : lock + (long)(q - nl) * n;
    double s0 = 0.0, s1 = 0.0;
    int k = lane;
    for (; k + 32 < n; k += 64) {
      s0 += x[k] * y[k];
      s1 += x[k + 32] * y[k + 32];
    }
    for (; k < n; k += 32) s0 += x[k] * y[k];
    double s = s0 + s1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[q] = s;
  }
  __syncthreads();
}

// number of eigenvalues of the tridiagonal (d, e) below x (Sturm count)
__device__ __forceinline__ int sturm(int m, const double* d, const double* e2, double x) {
  int c = 0;
  double q = d[0] - x;
  if (q < 0) ++c;
  for (int i = 1; i < m; ++i) {
    if (q == 0.0) q = 1e-300;
    q = d[i] - x - e2[i - 1] / q;
    if (q < 0) ++c;
  }
  return c;
}

// Solves (T - th I) y = b in place (b in y), T symmetric tridiagonal with
// diagonal al and off-diagonal bt: Gaussian elimination of the subdiagonal
// with a row interchange whenever the subdiagonal entry is the larger pivot
// (the interchange fills a second superdiagonal), then back substitution.
__host__ __device__ inline void tri_solve_pivoted(int m, const double* al, const double* bt,
                                                  double th, double* y) {
  double d[kEigMaxM], du[kEigMaxM], du2[kEigMaxM];
  for (int i = 0; i < m; ++i) {
    d[i] = al[i] - th;
    du[i] = i + 1 < m ? bt[i] : 0.0;
    du2[i] = 0.0;
  }
  for (int i = 0; i + 1 < m; ++i) {
    const double sub = bt[i];  // row i+1, column i
    if (fabs(d[i]) >= fabs(sub)) {
      if (d[i] == 0.0) d[i] = 1e-300;
      const double f = sub / d[i];
      d[i + 1] -= f * du[i];
      y[i + 1] -= f * y[i];
    } else {
      const double f = d[i] / sub;
      const double di1 = d[i + 1], dui1 = du[i + 1];
      d[i] = sub;
      d[i + 1] = du[i] - f * di1;
      du[i] = di1;
      du2[i] = dui1;
      du[i + 1] = -f * dui1;
      const double yi = y[i];
      y[i] = y[i + 1];
      y[i + 1] = yi - f * y[i + 1];
    }
  }
  if (d[m - 1] == 0.0) d[m - 1] = 1e-300;
  for (int i = m - 1; i >= 0; --i) {
    double s = y[i];
    if (i + 1 < m) s -= du[i] * y[i + 1];
    if (i + 2 < m) s -= du2[i] * y[i + 2];
    y[i] = s / d[i];
  }
}

}  // namespace

__global__ void __launch_bounds__(kEigThreads) eig_kernel(EigArgs a) {
  constexpr int NV = kEigMaxM + kEigMaxStates;
  __shared__ double ws[(kEigThreads / 32) * NV];
  __shared__ double red[NV];
  __shared__ double s_lk[kEigMaxStates];
  __shared__ double s_al[kEigMaxM], s_bt[kEigMaxM], s_e2[kEigMaxM], s_y[kEigMaxM];
  __shared__ double s_r[kEigMaxM];
  __shared__ double s_theta, s_bt0;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int p = blockIdx.x, n = a.n, m = a.m;
  const double* V = a.vpot + (long)p * n;
  double* L = a.L + (long)p * m * n;
  double* work = a.work + (long)p * n;

  for (int K = 0; K < a.nstates; ++K) {
    const double* st = a.start + ((long)p * a.nstates + K) * n;
    double* v = a.vec + ((long)p * a.nstates + K) * n;  // the current vector
    for (int k = t; k < n; k += kEigThreads) v[k] = st[k];
    __syncthreads();
    int count = 0;
    double res = 0.0;
    const double* lock = a.vec + (long)p * a.nstates * n;  // states 0..K-1
    for (int rs = 0; rs < a.maxrest; ++rs) {
      // ---- project the locked states out of v
      if (K > 0) {
        warp_dots(v, nullptr, 0, lock, K, n, red);
        for (int k = t; k < n; k += kEigThreads) {
          double vk = v[k];
          for (int j = 0; j < K; ++j) vk -= red[j] * lock[(long)j * n + k];
          v[k] = vk;
        }
        __syncthreads();
      }
      // ---- m Lanczos steps from v (lnz.f:76-119)
      {
        double acc[1] = {0.0};
        for (int k = t; k < n; k += kEigThreads) acc[0] += v[k] * v[k];
        cta_sums<1>(acc, 1, ws, red);
        if (t == 0) s_bt0 = sqrt(red[0]);
        __syncthreads();
      }
      for (int it = 0; it < m; ++it) {
        const double bt0 = s_bt0;
        const double* src = it == 0 ? v : work;
        double* Li = L + (long)it * n;
        for (int k = t; k < n; k += kEigThreads) Li[k] = src[k] / bt0;
        __syncthreads();
        // w = H vi - bt0 v_prev into work, al = <vi, w> (lnz.f:96-107)
        {
          double acc[1] = {0.0};
          for (int k = t; k < n; k += kEigThreads) {
            const double vp = it ? L[(long)(it - 1) * n + k] : 0.0;
            const double w = hx(a, V, Li, k, 1.0) - bt0 * vp;
            work[k] = w;
            acc[0] += Li[k] * w;
          }
          cta_sums<1>(acc, 1, ws, red);
          if (t == 0) s_al[it] = red[0];
          __syncthreads();
        }
        ++count;
        // work = w - al vi, then classical Gram-Schmidt against the locked
        // states and L_0..L_it (reort.f:65-80: all dot products, then all
        // updates): one pass for the dots, one for the updates and the norm
        const double al = s_al[it];
        for (int k = t; k < n; k += kEigThreads) work[k] = work[k] - al * Li[k];
        __syncthreads();
        warp_dots(work, L, it + 1, lock, K, n, red);
        if (t == 0) {
          for (int q = 0; q <= it; ++q) s_r[q] = red[q];
          for (int j = 0; j < K; ++j) s_lk[j] = red[it + 1 + j];
        }
        __syncthreads();
        double nn[1] = {0.0};
        for (int k = t; k < n; k += kEigThreads) {
          double w = work[k];
          for (int j = 0; j < K; ++j) w -= s_lk[j] * lock[(long)j * n + k];
          for (int q = 0; q <= it; ++q) w -= s_r[q] * L[(long)q * n + k];
          work[k] = w;
          nn[0] += w * w;
        }
        cta_sums<1>(nn, 1, ws, red);
        if (t == 0) {
          s_bt[it] = sqrt(red[0]);
          s_bt0 = s_bt[it];
        }
        __syncthreads();
      }
      // ---- lowest Ritz pair of T (DSTEVX('V','I',...,IL,IU))
      if (warp == 0) {
        if (lane == 0) {
          for (int i = 0; i + 1 < m; ++i) s_e2[i] = s_bt[i] * s_bt[i];
        }
        __syncwarp();
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < m; ++i) {  // Gershgorin interval
          const double r = (i > 0 ? fabs(s_bt[i - 1]) : 0.0) + (i + 1 < m ? fabs(s_bt[i]) : 0.0);
          lo = fmin(lo, s_al[i] - r);
          hi = fmax(hi, s_al[i] + r);
        }
        const double span = hi - lo;
        lo -= 1e-12 * span + 1e-300;
        hi += 1e-12 * span + 1e-300;
        // multisection: the K-th eigenvalue lies where the count passes K
        for (int round = 0; round < 16; ++round) {
          const double x = lo + (hi - lo) * (lane + 1) / 33.0;
          const int c = sturm(m, s_al, s_e2, x);
          const unsigned below = __ballot_sync(0xffffffffu, c <= 0);  // points below all
          const int nb = __popc(below);  // counts grow with x: the first nb points
          const double nlo = nb > 0 ? lo + (hi - lo) * nb / 33.0 : lo;
          const double nhi = nb < 32 ? lo + (hi - lo) * (nb + 1) / 33.0 : hi;
          lo = nlo;
          hi = nhi;
          if (hi - lo <= 4e-16 * fmax(fabs(lo), fabs(hi))) break;
        }
        if (lane == 0) {
          const double th = 0.5 * (lo + hi);
          s_theta = th;
          // inverse iteration on T - th I from a vector of ones, three
          // sweeps, each a tridiagonal solve with row interchanges
          double y[kEigMaxM];
          for (int i = 0; i < m; ++i) y[i] = 1.0;
          for (int sweep = 0; sweep < 3; ++sweep) {
            tri_solve_pivoted(m, s_al, s_bt, th, y);
            double nrm = 0.0;
            for (int i = 0; i < m; ++i) nrm += y[i] * y[i];
            nrm = sqrt(nrm);
            for (int i = 0; i < m; ++i) y[i] /= nrm;
          }
          for (int i = 0; i < m; ++i) s_y[i] = y[i];
        }
      }
      __syncthreads();
      // ---- v = L y, normalised (lanczsc.f:99-113, FATN = ECNORM)
      {
        double acc[1] = {0.0};
        for (int k = t; k < n; k += kEigThreads) {
          double s = 0.0;
          for (int j = 0; j < m; ++j) s += s_y[j] * L[(long)j * n + k];
          v[k] = s;
          acc[0] += s * s;
        }
        cta_sums<1>(acc, 1, ws, red);
        const double inv = 1.0 / sqrt(red[0]);
        for (int k = t; k < n; k += kEigThreads) v[k] *= inv;
        __syncthreads();
      }
      // ---- true residual |H v - theta v|
      {
        double acc[1] = {0.0};
        const double th = s_theta;
        for (int k = t; k < n; k += kEigThreads) {
          const double r = hx(a, V, v, k, 1.0) - th * v[k];
          acc[0] += r * r;
        }
        ++count;
        cta_sums<1>(acc, 1, ws, red);
        res = sqrt(red[0]);
      }
      if (res <= a.tol) break;
    }
    if (t == 0) {
      const long o = (long)p * a.nstates + K;
      a.eval[o] = s_theta;
      a.resid[o] = res;
      a.matvecs[o] = count;
    }
    __syncthreads();
  }
}

// LCG of rans.f:38-39 (NSEED = MOD(NSEED*1029 + 221591, 2^20), RAN = NSEED/2^20)
// jumped ahead: value number idx (1-based) of the sequence from seed 1
__global__ void lcg_kernel(double* out, long count, long first) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const unsigned long long M = 1ull << 20;
  // affine map f(x) = A x + C; f^j by binary powering
  unsigned long long A = 1, C = 0, bA = 1029, bC = 221591;
  unsigned long long e = (unsigned long long)(first + i);
  while (e) {
    if (e & 1) {  // (A, C) <- (bA, bC) o (A, C)
      C = (bA * C + bC) % M;
      A = (bA * A) % M;
    }
    bC = (bA * bC + bC) % M;
    bA = (bA * bA) % M;
    e >>= 1;
  }
  const unsigned long long x = (A * 1ull + C) % M;
  out[i] = (double)x / (double)M;
}

}  // namespace espec

using namespace espec;

#define EIG_CK(call)                                         \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_); \
  } while (0)

// 2D coupled Morse family (potfuncs.f:104-108 Morse terms plus a bilinear
// coupling): V = De1 (1 - e^{-a1 (x-re1)})^2 + De2 (1 - e^{-a2 (y-re2)})^2
// + lam (x-re1)(y-re2), params [nprob][5] = (De1, a1, De2, a2, lam)
__global__ void morse2d_kernel(const double* params, int nprob, int nx, int ny, double x0,
                               double hxs, double y0, double hys, double re1, double re2,
                               double* vpot) {
  const long n = (long)nx * ny;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n * nprob) return;
  const long p = gid / n, k = gid % n;
  const int i = (int)(k % nx), j = (int)(k / nx);
  const double x = x0 + i * hxs, y = y0 + j * hys;
  const double* q = params + p * 5;
  const double ex = 1.0 - exp(-q[1] * (x - re1)), ey = 1.0 - exp(-q[3] * (y - re2));
  vpot[gid] = q[0] * ex * ex + q[2] * ey * ey + q[4] * (x - re1) * (y - re2);
}

extern "C" int espec_eig_morse2d(int nprob, const double* params, const int* np, double xi,
                                 double xf, double yi, double yf, double re1, double re2,
                                 double* vpot, void* stream) {
  if (nprob <= 0 || !params || !np || !vpot || np[0] < 2 || np[1] < 2)
    return set_error(ESPEC_EINVAL, "bad argument");
  const long tot = (long)np[0] * np[1] * nprob;
  morse2d_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      params, nprob, np[0], np[1], xi, (xf - xi) / (np[0] - 1), yi, (yf - yi) / (np[1] - 1), re1,
      re2, vpot);
  EIG_CK(cudaGetLastError());
  return ESPEC_OK;
}

extern "C" int espec_eig_lcg_start(double* d_out, int n, int nstates, void* stream) {
  // lanczsc.f:56-62: N draws discarded, then N draws per state
  if (!d_out || n <= 0 || nstates <= 0) return set_error(ESPEC_EINVAL, "bad argument");
  const long count = (long)n * nstates;
  lcg_kernel<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_out, count,
                                                                               (long)n + 1);
  EIG_CK(cudaGetLastError());
  return ESPEC_OK;
}

extern "C" int espec_eig_solve_dev(int nprob, const int* np, const double* shm,
                                   const double* vpot, const double* start, int nstates, int m,
                                   double tol, int maxrest, double* vec, double* eval,
                                   double* resid, int* matvecs, double* work_L, double* work_v,
                                   void* stream) {
  if (nprob <= 0 || !np || !shm || !vpot || !start || !vec || !eval || !resid || !matvecs ||
      !work_L || !work_v)
    return set_error(ESPEC_EINVAL, "null argument");
  if (m < 2 || m > kEigMaxM) return set_error(ESPEC_EINVAL, "Lanczos length must be 2..48");
  if (nstates < 1 || nstates > kEigMaxStates) return set_error(ESPEC_EINVAL, "nstates must be 1..16");
  if (np[0] < 1 || np[1] < 1) return set_error(ESPEC_EINVAL, "bad grid");
  EigArgs a{};
  a.nx = np[0];
  a.ny = np[1];
  a.n = np[0] * np[1];
  a.shm[0] = shm[0];
  a.shm[1] = shm[1];
  a.sht30 = 30.0 * (shm[0] + shm[1]);
  a.vpot = vpot;
  a.start = start;
  a.L = work_L;
  a.work = work_v;
  a.vec = vec;
  a.eval = eval;
  a.resid = resid;
  a.matvecs = matvecs;
  a.nstates = nstates;
  a.m = m;
  a.maxrest = maxrest;
  a.tol = tol;
  eig_kernel<<<nprob, kEigThreads, 0, (cudaStream_t)stream>>>(a);
  EIG_CK(cudaGetLastError());
  return ESPEC_OK;
}
