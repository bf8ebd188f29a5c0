// spo1d_static.cu -- batched 1D split-operator propagation that allocates
// nothing.
//
// espec_spo_run_static() serves callers that may not allocate device memory
// at all: codes embedded in an application that owns the whole device
// memory pool (a Fortran driver that sized every array at start-up, a
// framework with its own caching allocator, a process that runs under a
// memory budget), and code running where cudaMalloc is forbidden, e.g. while
// another component is capturing or replaying work.  The caller passes
// device pointers for every input and output; all intermediate tables live in
// one file-scope __device__ array of fixed size (g_spo_static_scratch), so
// the call itself never calls cudaMalloc, cudaFree or any allocating library
// routine.  Every GPU that loads this library holds that array until the
// process exits.
//
// Limits: at most kStaticMaxPackets packets and kStaticMaxPoints grid points
// in total per call; no absorber and no reference-defect mode.
//
// Sharing: all calls use the same array, which keeps the contents of the
// last call.  Each call overwrites every scratch value it reads before
// reading it, so nothing has to start at zero.  Two calls whose GPU work
// overlaps (on different streams, or from different host threads) race on
// the array: serialise them.
//
// Set-up: the first call on each device resolves the array's device address
// with cudaGetSymbolAddress and caches it for that device (device code
// names the array directly, host code only passes the resolved pointer).
// Make that first call on each device before any stream capture begins.
// The cached address assumes one CUDA context per device for the life of the
// process (the runtime's primary context): after cudaDeviceReset the cache
// would hold a stale address, so a process that resets a device must not
// call this entry on it again.
#include <cuda_runtime.h>

#include "espec_gpu.h"
#include "espec_internal.h"
#include "spo1d_launch.cuh"

namespace espec {

constexpr int kStaticMaxPackets = 128;
constexpr int kStaticMaxPoints = 32768;
constexpr int kStaticMaxDevices = 64;

// per point: 5 FP64 tables (80 B) + kinetic table TC (8 B) + final-layout
// frequency (4 B) + packet id (4 B); per packet: descriptors and scalars
constexpr size_t kStaticPointBytes = 5 * sizeof(cpx<double>) + 8 + 4 + 4;
constexpr size_t kStaticPacketBytes = sizeof(SpoPacket) + 4 + 4 + 8 + 8 + 8 + 8;
constexpr size_t kStaticBytes =
    (size_t)kStaticMaxPoints * kStaticPointBytes + (size_t)(kStaticMaxPackets + 1) * kStaticPacketBytes + 1024;

static __device__ __align__(256) unsigned char g_spo_static_scratch[kStaticBytes];

// host-side cache of the resolved device address, one slot per device
static void* g_static_addr[kStaticMaxDevices];

// radices of DefaultPlan<N> (used to derive the final-layout frequencies)
struct StaticRadices {
  int n[8];     // size class
  int s[8];     // number of stages
  int r[8][8];  // radices
  int n3[8];    // unitary radix-3 stages
  int count;
};

template <class PL>
static void fill_radices(StaticRadices& sr, int i) {
  sr.n[i] = PL::N;
  sr.s[i] = PL::S;
  for (int k = 0; k < PL::S; ++k) sr.r[i][k] = PL::r[k];
  sr.n3[i] = PL::n3();
}

static bool static_size(int n, StaticRadices& sr, int i) {
  switch (n) {
    case 256: fill_radices<DefaultPlan<256>::type>(sr, i); return true;
    case 384: fill_radices<DefaultPlan<384>::type>(sr, i); return true;
    case 512: fill_radices<DefaultPlan<512>::type>(sr, i); return true;
    case 768: fill_radices<DefaultPlan<768>::type>(sr, i); return true;
    case 1024: fill_radices<DefaultPlan<1024>::type>(sr, i); return true;
    case 1536: fill_radices<DefaultPlan<1536>::type>(sr, i); return true;
    case 2048: fill_radices<DefaultPlan<2048>::type>(sr, i); return true;
    case 4096: fill_radices<DefaultPlan<4096>::type>(sr, i); return true;
    default: return false;
  }
}

struct StaticLayout {
  cpx<double>* tab;  // 5 * np entries (FP64) or the FP32 tables in the same bytes
  double* tc;
  int* kperm;
  int* pk_of;
  SpoPacket* pk;  // grouped by size class
  int* pk_off;
  int* npts;
  double* sh;
  double* sm;
  double* kscale;
};

static StaticLayout static_layout(unsigned char* base) {
  StaticLayout L;
  const size_t np = kStaticMaxPoints, nk = kStaticMaxPackets + 1;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base + o;
    o += (bytes + 255) / 256 * 256;
    return p;
  };
  L.tab = (cpx<double>*)take(np * 5 * sizeof(cpx<double>));
  L.tc = (double*)take(np * 8);
  L.kperm = (int*)take(np * 4);
  L.pk_of = (int*)take(np * 4);
  L.pk = (SpoPacket*)take(nk * sizeof(SpoPacket));
  L.pk_off = (int*)take(nk * 4);
  L.npts = (int*)take(nk * 4);
  L.sh = (double*)take(nk * 8);
  L.sm = (double*)take(nk * 8);
  L.kscale = (double*)take(nk * 8);
  return L;
}

// Per packet (one CTA each): packet ids, final-layout frequencies and the
// kinetic table of dkeft.f:64-79 (p accumulated by repeated addition, so one
// thread walks it in order).
__global__ void static_index_kernel(StaticLayout L, StaticRadices sr) {
  const int pk = blockIdx.x;
  const int n = L.npts[pk], base = L.pk_off[pk];
  int c = 0;
  while (c < sr.count && sr.n[c] != n) ++c;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    // kappa = k'_0 + R_0 (k'_1 + R_1 (...)) with digits of j from the outer stage
    int rem = j, M = n, f = 0, mult = 1;
    for (int s = 0; s < sr.s[c]; ++s) {
      const int R = sr.r[c][s], m = M / R;
      f += (rem / m) * mult;
      mult *= R;
      rem %= m;
      M = m;
    }
    L.kperm[base + j] = f;
    L.pk_of[base + j] = pk;
  }
  if (threadIdx.x == 0) {
    const double twopi = 6.283185307;  // dkeft.f:38
    const double sh = L.sh[pk], sm = L.sm[pk];
    const double dp = twopi / (n * sh);
    double p = 0.0;
    for (int i = 0; i < n / 2; ++i) {
      L.tc[base + i] = p * p / (2.0 * sm);
      p = p + dp;
    }
    p = -p;
    for (int i = n / 2; i < n; ++i) {
      L.tc[base + i] = p * p / (2.0 * sm);
      p = p + dp;
    }
  }
}

// Per point: e^{-iV dt}, e^{-iV dt/2}, kinetic phase in final layout, and the
// C(t) weight conj(psi0) e^{-iV dt/2} (no absorber), FP64 angle generation.
__global__ void static_table_kernel(StaticLayout L, const double* vpot, const double2* psi0,
                                    int npts, double cst1, double cst2, int fp32) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= npts) return;
  const int pk = L.pk_of[x];
  const int base = L.pk_off[pk];
  const double th = cst2 * vpot[x];
  double sh, ch, s2, c2, sk, ck;
  sincos(th, &sh, &ch);
  sincos(2.0 * th, &s2, &c2);
  const double tk = cst1 * L.tc[base + L.kperm[x]];
  sincos(tk, &sk, &ck);
  const double ks = L.kscale[pk];
  const double2 p0 = psi0[x];
  const double wr = p0.x * ch - p0.y * sh, wi = -p0.x * sh - p0.y * ch;
  const size_t np = kStaticMaxPoints;
  if (fp32) {
    auto ph = [](double phi, double a) {
      RotF r = make_rotf(phi);
      Tab<float>::phase_t o;
      o.t = r.t;
      o.s = r.s;
      o.ag = (float)(r.g * a);
      return o;
    };
    auto* t32 = reinterpret_cast<Tab<float>::phase_t*>(L.tab);
    t32[x] = ph(-2.0 * th, 1.0);
    t32[np + x] = ph(-th, 1.0);
    t32[2 * np + x] = ph(-th, 1.0);
    t32[3 * np + x] = ph(-tk, ks);
    reinterpret_cast<cpx<float>*>(t32 + 4 * np)[x] = mk((float)wr, (float)wi);
  } else {
    L.tab[x] = mk(c2, -s2);
    L.tab[np + x] = mk(ch, -sh);
    L.tab[2 * np + x] = mk(ch, -sh);
    L.tab[3 * np + x] = mk(ck * ks, -sk * ks);
    L.tab[4 * np + x] = mk(wr, wi);
  }
}

}  // namespace espec

using namespace espec;

extern "C" int espec_spo_run_static(int npk, const int* npts, const double* sh, const double* sm,
                                    double dt_fs, int precision, const double* vpot,
                                    const double* psi0, int nsteps, double* c_out,
                                    double* psi_out, void* stream) {
  if (npk <= 0 || !npts || !sh || !sm || !vpot || !psi0 || !c_out || nsteps < 0)
    return set_error(ESPEC_EINVAL, "espec_spo_run_static: null or invalid argument");
  if (precision != ESPEC_FP64 && precision != ESPEC_MIXED)
    return set_error(ESPEC_EINVAL, "espec_spo_run_static: precision must be ESPEC_FP64 or ESPEC_MIXED");
  if (npk > kStaticMaxPackets)
    return set_error(ESPEC_EINVAL, "espec_spo_run_static: more than 128 packets (static limit)");
  // host-side bookkeeping in fixed-size stack arrays only
  int off[kStaticMaxPackets + 1];
  double kscale[kStaticMaxPackets];
  SpoPacket pk[kStaticMaxPackets];
  StaticRadices sr{};
  off[0] = 0;
  for (int i = 0; i < npk; ++i) {
    int c = 0;
    while (c < sr.count && sr.n[c] != npts[i]) ++c;
    if (c == sr.count) {
      if (!static_size(npts[i], sr, c))
        return set_error(ESPEC_EINVAL, "espec_spo_run_static: unsupported packet size (supported: "
                                       "256, 384, 512, 768, 1024, 1536, 2048, 4096)");
      sr.count++;
    }
    double gain = npts[i];
    if (precision == ESPEC_MIXED)
      for (int k = 0; k < sr.n3[c]; ++k) gain /= 3.0;
    kscale[i] = 1.0 / gain;
    off[i + 1] = off[i] + npts[i];
    if (off[i + 1] > kStaticMaxPoints)
      return set_error(ESPEC_EINVAL,
                       "espec_spo_run_static: more than 32768 grid points in total (static limit)");
  }
  // packets grouped by size class, each class contiguous in pk[]
  int cls_first[8], cls_count[8], m = 0;
  for (int c = 0; c < sr.count; ++c) {
    cls_first[c] = m;
    cls_count[c] = 0;
    for (int i = 0; i < npk; ++i)
      if (npts[i] == sr.n[c]) {
        pk[m++] = SpoPacket{off[i], (long long)i * (nsteps + 1)};
        cls_count[c]++;
      }
  }
  // once per device: resolve the scratch array's address
  int dev = 0;
  int rc = ck(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= kStaticMaxDevices)
    return set_error(ESPEC_EINVAL, "espec_spo_run_static: device ordinal out of range");
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    rc = ck(cudaGetSymbolAddress(&p, g_spo_static_scratch), "cudaGetSymbolAddress");
    if (rc) return rc;
    g_static_addr[dev] = p;
  }
  cudaStream_t st = (cudaStream_t)stream;
  StaticLayout L = static_layout((unsigned char*)g_static_addr[dev]);
  const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
  if ((rc = ck(cudaMemcpyAsync(L.pk_off, off, sizeof(int) * (npk + 1), h2d, st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(L.npts, npts, sizeof(int) * npk, h2d, st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(L.sh, sh, sizeof(double) * npk, h2d, st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(L.sm, sm, sizeof(double) * npk, h2d, st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(L.kscale, kscale, sizeof(double) * npk, h2d, st), "H2D")) ||
      (rc = ck(cudaMemcpyAsync(L.pk, pk, sizeof(SpoPacket) * npk, h2d, st), "H2D")))
    return rc;
  static_index_kernel<<<npk, 256, 0, st>>>(L, sr);
  if ((rc = ck(cudaGetLastError(), "static_index_kernel"))) return rc;
  const int npts_total = off[npk];
  const double cst1 = dt_fs / ESPEC_SHFS, cst2 = dt_fs / (2.0 * ESPEC_SHFS);
  static_table_kernel<<<(npts_total + 255) / 256, 256, 0, st>>>(
      L, vpot, (const double2*)psi0, npts_total, cst1, cst2, precision == ESPEC_MIXED);
  if ((rc = ck(cudaGetLastError(), "static_table_kernel"))) return rc;
  const size_t np = kStaticMaxPoints;
  for (int c = 0; c < sr.count; ++c) {
    cudaError_t e;
    if (precision == ESPEC_FP64) {
      SpoArgs<double> a{};
      a.tab.g = L.tab;
      a.tab.h = L.tab + np;
      a.tab.hm = L.tab + 2 * np;
      a.tab.k = L.tab + 3 * np;
      a.tab.w = L.tab + 4 * np;
      a.pk = L.pk + cls_first[c];
      a.psi0 = (const double2*)psi0;
      a.psi_out = (double2*)psi_out;
      a.c_out = (double2*)c_out;
      a.nsteps = nsteps;
      e = (sr.n[c] & (sr.n[c] - 1)) == 0 ? spo_launch_f64_pow2(sr.n[c], 0, a, cls_count[c], false, st)
                                         : spo_launch_f64_r3(sr.n[c], 0, a, cls_count[c], false, st);
    } else {
      auto* t32 = reinterpret_cast<Tab<float>::phase_t*>(L.tab);
      SpoArgs<float> a{};
      a.tab.g = t32;
      a.tab.h = t32 + np;
      a.tab.hm = t32 + 2 * np;
      a.tab.k = t32 + 3 * np;
      a.tab.w = reinterpret_cast<cpx<float>*>(t32 + 4 * np);
      a.pk = L.pk + cls_first[c];
      a.psi0 = (const double2*)psi0;
      a.psi_out = (double2*)psi_out;
      a.c_out = (double2*)c_out;
      a.nsteps = nsteps;
      e = (sr.n[c] & (sr.n[c] - 1)) == 0 ? spo_launch_f32_pow2(sr.n[c], 0, a, cls_count[c], st)
                                         : spo_launch_f32_r3(sr.n[c], 0, a, cls_count[c], st);
    }
    if (e != cudaSuccess) return set_cuda_error("espec_spo_run_static launch", e);
  }
  return ESPEC_OK;
}
