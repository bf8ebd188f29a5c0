// potential.cu -- analytic potentials on the grid, on the GPU: the forms of
// POT1D / POT2D / POT3D (potfuncs.f:3-497) and the grid loop of GVPOT
// (gvpot.f:1-111) with its optional shift by the grid minimum.
//
// Batched 1D: one CTA per packet (a parameter scan: thousands of packets of
// uneven size, each with its own constants), the minimum found by a block
// reduction that keeps the first grid point holding it (GVPOT's strict "<"
// scan in grid order), then the shift.  2D/3D: one grid, V written by a
// grid-stride kernel, the minimum by per-CTA partials and one finishing CTA.
// Constants are those GVPOT receives: the deck's values after MAKECST, in
// atomic units (bohr, hartree, electron masses), 14 per potential (MXCST).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {
namespace {

constexpr int kCst = 14;  // MXCST (param.f)

// Every form keeps the association of the Fortran expression it restates
// (A*B**2/C is (A*(B*B))/C, left to right) and the file is compiled without
// FMA contraction, so a potential differs from the reference's only through
// the last bit of exp / cos.
__device__ __forceinline__ double sq(double v) { return v * v; }

__device__ double pot1d(int k, const double* c, double x) {
  switch (k) {
    case ESPEC_POT_OHS: return 0.5 * c[1] * sq(x - c[0]);
    case ESPEC_POT_DOHS:  // potfuncs.f:66-68 (exponent with a + sign, as written)
      return 0.5 * c[1] * sq(x - c[0]) + c[4] * exp(sq(x - c[2]) / sq(c[3]));
    case ESPEC_POT_MORSEM:
      return c[2] * (exp(-2.0 * c[1] * (x - c[0])) - 2.0 * exp(-c[1] * (x - c[0])));
    case ESPEC_POT_ANTI_MORSEM:
      return c[2] / 2.0 * (exp(-2.0 * c[1] * (x - c[0])) + 2.0 * exp(-c[1] * (x - c[0])));
    case ESPEC_POT_MOD_MORSE: return c[2] * sq(c[3] - exp(-c[1] * (x - c[0]))) + c[4];
    case ESPEC_POT_MORSE: return c[2] * sq(1.0 - exp(-c[1] * (x - c[0])));
    case ESPEC_POT_ANTI_MORSE: return c[2] / 2.0 * sq(1.0 + exp(-c[1] * (x - c[0])));
    case ESPEC_POT_DMORSE:
      return c[2] * sq(1.0 - exp(-c[3] * (x - c[0]))) + c[4] * exp(-(c[5] * sq(x - c[1])));
    case ESPEC_POT_STEP: return (x >= c[0] && x <= c[1]) ? 0.0 : c[2];
    case ESPEC_POT_BARRIER: return (x >= c[0] && x <= c[1]) ? c[2] : 0.0;
    default: return c[0];  // ESPEC_POT_CONST (.CONST / .FREE)
  }
}

// LEPS surface of three Sato-modified Morse pairs (potfuncs.f:433-487)
__device__ double leps(const double* c, double x, double y, double z) {
  const double a = c[9], b = c[10], g = c[11];
  const double m1 = pot1d(ESPEC_POT_MORSEM, c, x), s1 = pot1d(ESPEC_POT_ANTI_MORSEM, c, x);
  const double m2 = pot1d(ESPEC_POT_MORSEM, c + 3, y), s2 = pot1d(ESPEC_POT_ANTI_MORSEM, c + 3, y);
  const double m3 = pot1d(ESPEC_POT_MORSEM, c + 6, z), s3 = pot1d(ESPEC_POT_ANTI_MORSEM, c + 6, z);
  const double fa = (1 - a) / (1 + a), fb = (1 - b) / (1 + b), fg = (1 - g) / (1 + g);
  const double q1 = 0.5 * (m1 + fa * s1), q2 = 0.5 * (m2 + fb * s2), q3 = 0.5 * (m3 + fg * s3);
  const double j1 = 0.5 * (m1 - fa * s1), j2 = 0.5 * (m2 - fb * s2), j3 = 0.5 * (m3 - fg * s3);
  return q1 + q2 + q3 - sqrt(j1 * j1 + j2 * j2 + j3 * j3 - j1 * j2 - j2 * j3 - j1 * j3);
}

__device__ double pot3d(int k, const double* c, double x, double y, double z) {
  switch (k) {
    case ESPEC_POT_OHS:
      return 0.5 * c[1] * sq(x - c[0]) + 0.5 * c[3] * sq(y - c[2]) + 0.5 * c[5] * sq(z - c[4]);
    case ESPEC_POT_STEP:
      return (x >= c[0] && x <= c[1] && y >= c[2] && y <= c[3] && z >= c[4] && z <= c[5]) ? 0.0
                                                                                           : c[6];
    case ESPEC_POT_BARRIER:  // potfuncs.f:425-431 tests y against the z bounds, as written
      return (x >= c[0] && x <= c[1] && y >= c[2] && y <= c[3] && y >= c[4] && y <= c[5]) ? c[6]
                                                                                           : 0.0;
    case ESPEC_POT_LEPS: case ESPEC_POT_LEPS_CC: return leps(c, x, y, z);
    default: return c[0];
  }
}

__device__ double pot2d(int k, const double* sm, const double* c, double x, double y) {
  switch (k) {
    case ESPEC_POT_OHS: return 0.5 * c[1] * sq(x - c[0]) + 0.5 * c[3] * sq(y - c[2]);
    case ESPEC_POT_MORSE:
      return c[2] * sq(1.0 - exp(-c[1] * (x - c[0]))) + c[5] * sq(1.0 - exp(-c[4] * (y - c[3])));
    case ESPEC_POT_LSM: case ESPEC_POT_LS: {
      const double va = c[2] * (1.0 - exp(-(c[1] * sq(x - c[0]) / (2.0 * x + 1.0e-99))));
      const double vb =
          c[4] * (1.0 - exp(-(c[3] * sq(y - x - c[0]) / (2.0 * (y - c[0]) + 1.0e-99))));
      if (k == ESPEC_POT_LS) return va + vb;
      // potfuncs.f:221: the well depth is CST(2), as written
      return va + vb + c[1] * sq(1.0 - exp(-c[6] * (y - c[5])));
    }
    case ESPEC_POT_LBH_CC: case ESPEC_POT_LBH: {
      double rx = x, ry = y;
      if (k == ESPEC_POT_LBH_CC) {
        ry = y / sqrt(sm[1] * sm[2] * (sm[0] + sm[1] + sm[2]) /
                      ((sm[1] + sm[2]) * (sm[1] + sm[2]) * sm[0]));
        rx = x + sm[1] * ry / (sm[1] + sm[2]) - ry;
      }
      return c[0] * exp(-1.0 / c[1] * rx) +
             c[2] * (exp(-2.0 * c[3] * (ry - c[4])) - 2.0 * exp(-c[3] * (ry - c[4])));
    }
    case ESPEC_POT_LEPS_CC: {
      const double ry = y / sqrt(sm[1] * sm[2] * (sm[0] + sm[1] + sm[2]) /
                                 ((sm[1] + sm[2]) * (sm[1] + sm[2]) * sm[0]));
      const double rx = x - sm[1] * ry / (sm[1] + sm[2]);
      const double rz = sqrt(rx * rx + ry * ry - 2.0 * rx * ry * cos(c[12]));
      return leps(c, rx, ry, rz);
    }
    case ESPEC_POT_LEPS: {
      const double rz = sqrt(x * x + y * y - 2.0 * x * y * cos(c[12]));
      return leps(c, x, y, rz);
    }
    case ESPEC_POT_WELLXY:
      return ((x >= c[0] && x <= c[1]) ? 0.0 : c[2]) + ((y >= c[3] && y <= c[4]) ? 0.0 : c[5]);
    case ESPEC_POT_WELLX: return (x >= c[0] && x <= c[1]) ? 0.0 : c[2];
    case ESPEC_POT_WELLY: return (y >= c[0] && y <= c[1]) ? 0.0 : c[2];
    case ESPEC_POT_WELL:
      return (x >= c[0] && x <= c[1] && y >= c[2] && y <= c[3]) ? 0.0 : c[4];
    case ESPEC_POT_BARRIERXY:
      return ((x >= c[0] && x <= c[1]) ? c[2] : 0.0) + ((y >= c[3] && y <= c[4]) ? c[5] : 0.0);
    case ESPEC_POT_BARRIERX: return (x >= c[0] && x <= c[1]) ? c[2] : 0.0;
    case ESPEC_POT_BARRIERY: return (y >= c[0] && y <= c[1]) ? c[2] : 0.0;
    case ESPEC_POT_BARRIER:
      return (x >= c[0] && x <= c[1] && y >= c[2] && y <= c[3]) ? c[4] : 0.0;
    default: return c[0];
  }
}

// (value, grid index) with the smaller value, the first index on ties
struct VMin {
  double v;
  long i;
};
__device__ __forceinline__ VMin vmin(VMin a, VMin b) {
  return (b.v < a.v || (b.v == a.v && b.i < a.i)) ? b : a;
}

template <int NT>
__device__ VMin block_min(VMin m, VMin* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    VMin b{__shfl_xor_sync(0xffffffffu, m.v, o), __shfl_xor_sync(0xffffffffu, m.i, o)};
    m = vmin(m, b);
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < NT / 32 ? sh[threadIdx.x] : VMin{DBL_MAX, -1};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      VMin b{__shfl_xor_sync(0xffffffffu, m.v, o), __shfl_xor_sync(0xffffffffu, m.i, o)};
      m = vmin(m, b);
    }
  }
  return m;  // valid in thread 0
}

constexpr int kPotThreads = 256;

// grid coordinate XI + (I-1) SH with the product rounded before the sum, as
// the reference's Fortran computes it (a fused multiply-add would differ in
// the last bit, and XMIN with it)
__device__ __forceinline__ double coord(double xi, long i, double h) {
  return __dadd_rn(xi, __dmul_rn((double)i, h));
}

struct Gv1 {
  const int* off;    // [npk + 1] first point of each packet
  const double* xi;  // [npk]
  const double* sh;  // [npk]
  const double* cst; // [npk][kCst]
  int kind, shiftp;
  double* vpot;
  double* xmin;      // [npk]
};

// gvpot.f:21-34: RX = XI + (I-1) SH; the shift when the minimum is above 1e-6
__global__ void __launch_bounds__(kPotThreads) gvpot1d_kernel(Gv1 a) {
  __shared__ VMin sh[kPotThreads / 32];
  __shared__ double s_min;
  const int pk = blockIdx.x;
  const long o = a.off[pk], n = a.off[pk + 1] - o;
  const double* c = a.cst + (size_t)pk * kCst;
  const double xi = a.xi[pk], h = a.sh[pk];
  VMin m{DBL_MAX, -1};
  for (long i = threadIdx.x; i < n; i += kPotThreads) {
    const double v = pot1d(a.kind, c, coord(xi, i, h));
    a.vpot[o + i] = v;
    m = vmin(m, VMin{v, i});
  }
  m = block_min<kPotThreads>(m, sh);
  if (threadIdx.x == 0) {
    s_min = m.v;
    if (a.xmin) a.xmin[pk] = a.shiftp ? coord(xi, m.i, h) : 0.0;
  }
  __syncthreads();
  if (a.shiftp && s_min > 1.0e-6)
    for (long i = threadIdx.x; i < n; i += kPotThreads) a.vpot[o + i] -= s_min;
}

struct GvN {
  int ndim, nx, ny, nz;
  long n;
  double xi[3], sh[3], sm[3];
  double cst[kCst];
  int kind, quirk3d;
  double* vpot;
  VMin* part;   // [gridDim.x]
  double* vmin; // [1]
};

// gvpot.f:35-107, x fastest; the 3D loop takes RX from the z index
// (gvpot.f:96) when quirk3d is set
__global__ void __launch_bounds__(kPotThreads) gvpotnd_kernel(GvN a) {
  __shared__ VMin sh[kPotThreads / 32];
  VMin m{DBL_MAX, -1};
  for (long l = blockIdx.x * (long)kPotThreads + threadIdx.x; l < a.n;
       l += (long)gridDim.x * kPotThreads) {
    const long i = l % a.nx, j = (l / a.nx) % a.ny, k = l / ((long)a.nx * a.ny);
    double v;
    if (a.ndim == 2) {
      v = pot2d(a.kind, a.sm, a.cst, coord(a.xi[0], i, a.sh[0]), coord(a.xi[1], j, a.sh[1]));
    } else {
      const double rx = coord(a.xi[0], a.quirk3d ? k : i, a.sh[0]);
      v = pot3d(a.kind, a.cst, rx, coord(a.xi[1], j, a.sh[1]), coord(a.xi[2], k, a.sh[2]));
    }
    a.vpot[l] = v;
    m = vmin(m, VMin{v, l});
  }
  m = block_min<kPotThreads>(m, sh);
  if (threadIdx.x == 0) a.part[blockIdx.x] = m;
}

__global__ void __launch_bounds__(kPotThreads) gvpot_min_kernel(const VMin* part, int np,
                                                                 double* out) {
  __shared__ VMin sh[kPotThreads / 32];
  VMin m{DBL_MAX, -1};
  for (int i = threadIdx.x; i < np; i += kPotThreads) m = vmin(m, part[i]);
  m = block_min<kPotThreads>(m, sh);
  if (threadIdx.x == 0) *out = m.v;
}

// 2D: shift when |min| > 1e-6 (gvpot.f:64); 3D: when min > 1e-6 (gvpot.f:102)
__global__ void gvpot_shift_kernel(double* v, long n, const double* vmin, int ndim) {
  const double m = *vmin;
  const bool on = ndim == 2 ? fabs(m) > 1.0e-6 : m > 1.0e-6;
  if (!on) return;
  for (long l = blockIdx.x * (long)blockDim.x + threadIdx.x; l < n; l += (long)gridDim.x * blockDim.x)
    v[l] -= m;
}

}  // namespace
}  // namespace espec

using namespace espec;

// The reference's choice of form for POTCH (potfuncs.f): the first prefix
// test that matches, in the order of POT1D / POT2D / POT3D.
extern "C" int espec_pot_kind(const char* potch, size_t len, int ndim) {
  if (!potch) return 0;
  auto is = [&](const char* p) {
    const size_t k = std::strlen(p);
    return len >= k && std::strncmp(potch, p, k) == 0;
  };
  if (ndim == 1) {
    if (is(".OHS")) return ESPEC_POT_OHS;
    if (is(".DOHS")) return ESPEC_POT_DOHS;
    if (is(".MORSEM")) return ESPEC_POT_MORSEM;
    if (is(".ANTI-MORSEM")) return ESPEC_POT_ANTI_MORSEM;
    if (is(".MOD-MORSE")) return ESPEC_POT_MOD_MORSE;
    if (is(".MORSE")) return ESPEC_POT_MORSE;
    if (is(".ANTI-MORSE")) return ESPEC_POT_ANTI_MORSE;
    if (is(".DMORSE")) return ESPEC_POT_DMORSE;
    if (is(".STEP")) return ESPEC_POT_STEP;
    if (is(".BARRIER")) return ESPEC_POT_BARRIER;
    if (is(".CONST") || is(".FREE")) return ESPEC_POT_CONST;
    return 0;
  }
  if (ndim == 2) {
    if (is(".OHS")) return ESPEC_POT_OHS;
    if (is(".MORSE")) return ESPEC_POT_MORSE;
    if (is(".LSM")) return ESPEC_POT_LSM;
    if (is(".LS")) return ESPEC_POT_LS;
    if (is(".LBH_CC")) return ESPEC_POT_LBH_CC;
    if (is(".LBH")) return ESPEC_POT_LBH;
    if (is(".LEPS_CC")) return ESPEC_POT_LEPS_CC;
    if (is(".LEPS")) return ESPEC_POT_LEPS;
    if (is(".WELLXY")) return ESPEC_POT_WELLXY;
    if (is(".WELLX")) return ESPEC_POT_WELLX;
    if (is(".WELLY")) return ESPEC_POT_WELLY;
    if (is(".WELL")) return ESPEC_POT_WELL;
    if (is(".BARRIERXY")) return ESPEC_POT_BARRIERXY;
    if (is(".BARRIERX")) return ESPEC_POT_BARRIERX;
    if (is(".BARRIERY")) return ESPEC_POT_BARRIERY;
    if (is(".BARRIER")) return ESPEC_POT_BARRIER;
    if (is(".CONST") || is(".FREE")) return ESPEC_POT_CONST;
    return 0;
  }
  if (ndim == 3) {
    if (is(".OHS")) return ESPEC_POT_OHS;
    if (is(".STEP")) return ESPEC_POT_STEP;
    if (is(".BARRIER")) return ESPEC_POT_BARRIER;
    if (is(".LEPS")) return ESPEC_POT_LEPS;
    if (is(".CONST") || is(".FREE")) return ESPEC_POT_CONST;
  }
  return 0;
}

static bool kind_ok(int kind, int ndim) {
  if (ndim == 1) return kind >= ESPEC_POT_OHS && kind <= ESPEC_POT_CONST;
  if (ndim == 2)
    return kind == ESPEC_POT_OHS || kind == ESPEC_POT_MORSE || kind == ESPEC_POT_BARRIER ||
           kind == ESPEC_POT_CONST || (kind >= ESPEC_POT_LSM && kind <= ESPEC_POT_BARRIERY);
  return kind == ESPEC_POT_OHS || kind == ESPEC_POT_STEP || kind == ESPEC_POT_BARRIER ||
         kind == ESPEC_POT_LEPS || kind == ESPEC_POT_CONST;
}

extern "C" int espec_gvpot_1d(int npk, const int* npts, const double* xi, const double* sh,
                              int kind, const double* cst, int shiftp, double* vpot, double* xmin,
                              void* stream) {
  if (npk <= 0 || !npts || !xi || !sh || !cst || !vpot)
    return set_error(ESPEC_EINVAL, "espec_gvpot_1d: null or invalid argument");
  if (!kind_ok(kind, 1)) return set_error(ESPEC_EINVAL, "espec_gvpot_1d: not a POT1D form");
  cudaStream_t st = (cudaStream_t)stream;
  // one device block for the packet offsets, origins, steps, constants and xmin
  const size_t nb = sizeof(int) * (npk + 1) + sizeof(double) * ((size_t)npk * (3 + kCst));
  void* d = nullptr;
  int rc = ck(cudaMallocAsync(&d, nb, st), "cudaMallocAsync");
  if (rc) return rc;
  double* dd = (double*)d;
  double* d_xi = dd;
  double* d_sh = dd + npk;
  double* d_xmin = dd + 2 * (size_t)npk;
  double* d_cst = dd + 3 * (size_t)npk;
  int* d_off = (int*)(d_cst + (size_t)npk * kCst);
  // host staging: offsets as int prefix sums
  int* off = new int[npk + 1];
  off[0] = 0;
  for (int i = 0; i < npk; ++i) {
    if (npts[i] < 1 || (long long)off[i] + npts[i] > 0x7fffffff) {
      delete[] off;
      cudaFreeAsync(d, st);
      return set_error(ESPEC_EINVAL, "espec_gvpot_1d: bad packet size");
    }
    off[i + 1] = off[i] + npts[i];
  }
  cudaError_t e = cudaMemcpyAsync(d_xi, xi, sizeof(double) * npk, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_sh, sh, sizeof(double) * npk, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_cst, cst, sizeof(double) * npk * kCst, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, off, sizeof(int) * (npk + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    Gv1 a{d_off, d_xi, d_sh, d_cst, kind, shiftp ? 1 : 0, vpot, d_xmin};
    gvpot1d_kernel<<<npk, kPotThreads, 0, st>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && xmin)
    e = cudaMemcpyAsync(xmin, d_xmin, sizeof(double) * npk, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host staging is released below
  delete[] off;
  cudaFreeAsync(d, st);
  if (e != cudaSuccess) return set_cuda_error("espec_gvpot_1d", e);
  return ESPEC_OK;
}

extern "C" int espec_gvpot_nd(int ndim, const int* np, const double* xi, const double* sh,
                              const double* sm, int kind, const double* cst, int shiftp,
                              int quirks, double* vpot, void* stream) {
  if ((ndim != 2 && ndim != 3) || !np || !xi || !sh || !cst || !vpot)
    return set_error(ESPEC_EINVAL, "espec_gvpot_nd: null or invalid argument");
  if (!kind_ok(kind, ndim)) return set_error(ESPEC_EINVAL, "espec_gvpot_nd: not a form of this dimension");
  GvN a{};
  a.ndim = ndim;
  a.nx = np[0];
  a.ny = np[1];
  a.nz = ndim == 3 ? np[2] : 1;
  if (a.nx < 1 || a.ny < 1 || a.nz < 1) return set_error(ESPEC_EINVAL, "espec_gvpot_nd: bad grid");
  a.n = (long)a.nx * a.ny * a.nz;
  for (int d = 0; d < ndim; ++d) {
    a.xi[d] = xi[d];
    a.sh[d] = sh[d];
  }
  // the three masses SM(1..3) of the mass-scaled forms (.LBH_CC, .LEPS_CC)
  for (int d = 0; d < 3; ++d) a.sm[d] = sm ? sm[d] : 1.0;
  std::memcpy(a.cst, cst, sizeof(a.cst));
  a.kind = kind;
  a.quirk3d = (quirks & ESPEC_Q_GVPOT_3D) ? 1 : 0;
  a.vpot = vpot;
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = (int)std::min<long>((a.n + kPotThreads - 1) / kPotThreads, 148L * 8);
  void* d = nullptr;
  int rc = ck(cudaMallocAsync(&d, sizeof(VMin) * blocks + sizeof(double), st), "cudaMallocAsync");
  if (rc) return rc;
  a.part = (VMin*)d;
  a.vmin = (double*)(a.part + blocks);
  gvpotnd_kernel<<<blocks, kPotThreads, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && shiftp) {
    gvpot_min_kernel<<<1, kPotThreads, 0, st>>>(a.part, blocks, a.vmin);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      gvpot_shift_kernel<<<blocks, kPotThreads, 0, st>>>(vpot, a.n, a.vmin, ndim);
      e = cudaGetLastError();
    }
  }
  cudaFreeAsync(d, st);
  if (e != cudaSuccess) return set_cuda_error("espec_gvpot_nd", e);
  return ESPEC_OK;
}
