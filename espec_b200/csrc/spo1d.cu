// spo1d.cu -- batched 1D split-operator plans: table set-up, launches and
// the C-ABI entry points declared in include/espec_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"
#include "cplx_io.cuh"
#include "diag1d.cuh"
#include "sod1d.cuh"
#include "spo1d_any.cuh"
#include "spo1d_launch.cuh"
#include "spo1d_persist.cuh"

namespace espec {

// ---------------------------------------------------------------------------
// host-side index logic
// ---------------------------------------------------------------------------
// Frequency (FFT-order index) held at each final position of the DIF sequence
// of plan PL: kappa_M(j) = R * kappa_{M/R}(j mod M/R) + j / (M/R).
template <class PL>
static std::vector<int> final_freq() {
  std::vector<int> kap(PL::N);
  for (int j = 0; j < PL::N; ++j) {
    int f = 0, mult = 1, rem = j, M = PL::N;
    // unroll the recursion from the outermost stage
    std::vector<int> digits;
    for (int s = 0; s < PL::S; ++s) {
      const int R = PL::r[s];
      const int m = M / R;
      digits.push_back(rem / m);
      rem = rem % m;
      M = m;
    }
    // kappa = k'_0 + R_0 (k'_1 + R_1 (k'_2 + ...))
    for (int s = 0; s < PL::S; ++s) {
      f += digits[s] * mult;
      mult *= PL::r[s];
    }
    kap[j] = f;
  }
  return kap;
}

// dkeft.f:64-79 (DIGT, 1D): TC(k) = p^2 / (2 m) in FFT order with the
// reference's truncated 2 pi and p accumulated by repeated addition.
void digt_1d(int n, double sh, double sm, double* tc) {
  const double twopi = 6.283185307;
  const double dp = twopi / (n * sh);
  double p = 0.0;
  for (int i = 0; i < n / 2; ++i) {
    tc[i] = p * p / (2.0 * sm);
    p = p + dp;
  }
  p = -p;
  for (int i = n / 2; i < n; ++i) {
    tc[i] = p * p / (2.0 * sm);
    p = p + dp;
  }
}

// ---------------------------------------------------------------------------
// set-up kernel: FP64 phase generation with one argument reduction per value
// ---------------------------------------------------------------------------
struct SetupArgs {
  const double* vpot;
  const double* vabc;
  const double2* psi0;
  const double* tc;    // FFT order per packet
  const int* kperm;    // per point: FFT index held at this final position
  const int* pk_of;    // packet index of each point
  const int* pk_off;   // first point of each packet
  const double* kscale;  // per packet scale of the kinetic table
  int npts;
  double cst1, cst2;   // dt/SHFS, dt/(2 SHFS)
  int absorb;          // ESPEC_ABS_*
  int fp32;
  // outputs (one of the two sets)
  cpx<double>* g64;
  cpx<double>* h64;
  cpx<double>* hm64;
  cpx<double>* k64;
  cpx<double>* w64;
  Tab<float>::phase_t* g32;
  Tab<float>::phase_t* h32;
  Tab<float>::phase_t* hm32;
  Tab<float>::phase_t* k32;
  cpx<float>* w32;
  double* kq_c;
  double* kq_s;
};

__device__ __forceinline__ Tab<float>::phase_t phase32(double phi, double a) {
  RotF r = make_rotf(phi);
  Tab<float>::phase_t o;
  o.t = r.t;
  o.s = r.s;
  o.ag = (float)(r.g * a);
  return o;
}

__global__ void spo_setup_kernel(SetupArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.npts) return;
  const int pk = a.pk_of[x];
  const int base = a.pk_off[pk];
  // x-space factors.  h = e^{-i cst2 V} (x e^{cst2 VABC} for .VOPTIC)
  const double th = a.cst2 * a.vpot[x];
  double hmag = 1.0, mask = 1.0;
  if (a.absorb == ESPEC_ABS_VOPTIC) hmag = exp(a.cst2 * a.vabc[x]);
  if (a.absorb == ESPEC_ABS_SMOOTHW) mask = a.vabc[x];
  double sh, ch, s2, c2;
  sincos(th, &sh, &ch);
  sincos(2.0 * th, &s2, &c2);
  const double gmag = hmag * hmag * mask;
  const double2 p0 = a.psi0[x];
  // w = conj(psi0) * mask * h
  const double hr = ch * hmag * mask, hi = -sh * hmag * mask;
  const double wr = p0.x * hr + p0.y * hi, wi = p0.x * hi - p0.y * hr;
  // kinetic factor at this final position
  const int f = x - base;
  const int kidx = base + a.kperm[x];
  const double tk = a.cst1 * a.tc[kidx];
  double sk, ck;
  sincos(tk, &sk, &ck);
  const double ks = a.kscale[pk];
  if (a.fp32) {
    a.g32[x] = phase32(-2.0 * th, gmag);
    a.h32[x] = phase32(-th, hmag);
    a.hm32[x] = phase32(-th, hmag * mask);
    a.k32[x] = phase32(-tk, ks);
    a.w32[x] = mk((float)wr, (float)wi);
  } else {
    a.g64[x] = mk(c2 * gmag, -s2 * gmag);
    a.h64[x] = mk(ch * hmag, -sh * hmag);
    a.hm64[x] = mk(ch * hmag * mask, -sh * hmag * mask);
    a.k64[x] = mk(ck * ks, -sk * ks);
    a.w64[x] = mk(wr, wi);
    if (a.kq_c) {
      a.kq_c[x] = ck;
      a.kq_s[x] = sk;
    }
  }
  (void)f;
}

// SOD (.PFSOD) tables: CST V, CST TC/N (final layout), CST VABC or mask, conj(psi0)
__global__ void sod_setup_kernel(SetupArgs a, SodTables out, double cst) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= a.npts) return;
  const int pk = a.pk_of[x];
  const int base = a.pk_off[pk];
  const_cast<double*>(out.vc)[x] = cst * a.vpot[x];
  const_cast<double*>(out.kc)[x] = cst * a.tc[base + a.kperm[x]] * a.kscale[pk];
  if (a.absorb == ESPEC_ABS_VOPTIC) const_cast<double*>(out.ab)[x] = cst * a.vabc[x];
  if (a.absorb == ESPEC_ABS_SMOOTHW) const_cast<double*>(out.ab)[x] = a.vabc[x];
  const double2 p0 = a.psi0[x];
  const_cast<cpx<double>*>(out.w)[x] = mk(p0.x, -p0.y);
}

cudaError_t sod_launch(int n, int kabs, const SodArgs& a, int nblocks, cudaStream_t st);
bool sod_size_supported(int n);


// ---------------------------------------------------------------------------
// per-size-class dispatch
// ---------------------------------------------------------------------------
static bool size_supported(int n) {
  switch (n) {
    case 256: case 384: case 512: case 768: case 1024: case 1536: case 2048: case 4096:
      return true;
    default:
      return false;
  }
}

static bool is_pow2(int n) { return (n & (n - 1)) == 0; }

template <typename R>
static cudaError_t launch_n(int n, int v, const SpoArgs<R>& a, int nblocks, bool quirk,
                            cudaStream_t st) {
  if constexpr (sizeof(R) == 4) {
    return is_pow2(n) ? spo_launch_f32_pow2(n, v, a, nblocks, st)
                      : spo_launch_f32_r3(n, v, a, nblocks, st);
  } else {
    return is_pow2(n) ? spo_launch_f64_pow2(n, v, a, nblocks, quirk, st)
                      : spo_launch_f64_r3(n, v, a, nblocks, quirk, st);
  }
}

template <class PL>
static void fill_plan_info(std::vector<int>& kap, int& n3) {
  kap = final_freq<PL>();
  n3 = PL::n3();
}

template <int N>
static void plan_info_n(int v, std::vector<int>& kap, int& n3) {
  switch (v) {
    case 2: case 3: fill_plan_info<typename ClassicPlan<N>::type>(kap, n3); break;
    case 4: fill_plan_info<typename AltPlan<N>::type>(kap, n3); break;
    default: fill_plan_info<typename DefaultPlan<N>::type>(kap, n3); break;
  }
}

// final-layout frequencies and radix-3 count of the plan behind variant v
// the tensor-core variant of 256-point packets (spo_tc.cu)
void spo_tc256_final_freq(int* kap);
cudaError_t spo_tc256_launch(const SpoArgs<float>& a, int npk, cudaStream_t st);
int spo_tc_status(int* timed_out);

static void plan_info(int n, int v, std::vector<int>& kap, int& n3) {
  if (v == ESPEC_VARIANT_TC) {  // n == 256, mixed: no radix-3 stage
    kap.assign(256, 0);
    spo_tc256_final_freq(kap.data());
    n3 = 0;
    return;
  }
  switch (n) {
    case 256: plan_info_n<256>(v, kap, n3); break;
    case 384: plan_info_n<384>(v, kap, n3); break;
    case 512: plan_info_n<512>(v, kap, n3); break;
    case 768: plan_info_n<768>(v, kap, n3); break;
    case 1024: plan_info_n<1024>(v, kap, n3); break;
    case 1536: plan_info_n<1536>(v, kap, n3); break;
    case 2048: plan_info_n<2048>(v, kap, n3); break;
    case 4096: plan_info_n<4096>(v, kap, n3); break;
    default:  // the any-size kernels: natural order
      kap.resize(n);
      for (int j = 0; j < n; ++j) kap[j] = j;
      n3 = 0;
      break;
  }
}

static size_t smem_of(int n, int v, int precision) {
  const bool d = precision == ESPEC_FP64;
  switch (n) {
    case 256: return d ? variant_smem<double, 256>(v) : variant_smem<float, 256>(v);
    case 384: return d ? variant_smem<double, 384>(v) : variant_smem<float, 384>(v);
    case 512: return d ? variant_smem<double, 512>(v) : variant_smem<float, 512>(v);
    case 768: return d ? variant_smem<double, 768>(v) : variant_smem<float, 768>(v);
    case 1024: return d ? variant_smem<double, 1024>(v) : variant_smem<float, 1024>(v);
    case 1536: return d ? variant_smem<double, 1536>(v) : variant_smem<float, 1536>(v);
    case 2048: return d ? variant_smem<double, 2048>(v) : variant_smem<float, 2048>(v);
    case 4096: return d ? variant_smem<double, 4096>(v) : variant_smem<float, 4096>(v);
    default: return 0;
  }
}

static bool variant_fits(int n, int v, int precision) {
  const size_t b = smem_of(n, v, precision);
  return b > 0 && b <= kMaxSmem;
}

// default variant per size and precision: the fastest of espec_b200.autotune
// on B200 (300 time steps, >= 8 waves of CTAs per size)
static int default_variant(int n, int precision) {
  if (precision == ESPEC_MIXED) {
    switch (n) {
      case 256: return 1;
      case 384: return 2;
      case 512: return 3;
      case 768: return 2;
      case 1024: return 1;
      case 1536: return 2;
      case 2048: return 0;
      case 4096: return 2;
      default: return 0;
    }
  }
  switch (n) {
    case 256: case 384: case 512: case 768: case 4096: return 2;
    case 2048: return 1;
    default: return 0;
  }
}

}  // namespace espec

// ---------------------------------------------------------------------------
// plan object behind the C-ABI
// ---------------------------------------------------------------------------
using namespace espec;

struct espec_spo_plan {
  int npk = 0, npts = 0, precision = 0, absorb = 0, quirks = 0, method = ESPEC_SPO;
  double2* d_psi_prev = nullptr;  // SOD: psi(TF - dt)
  SodTables tsod{};
  double dt_fs = 0.0;
  std::vector<int> n, off;
  std::vector<double> sh, sm;
  struct Class {
    int n;
    int count;
    SpoPacket* d_pk;
    int variant;
    SpoPacket* d_pkd;  // diagnostics: c_off = packet index
    int* d_kfreq;      // FFT index at each final position of the diagnostic FFT
    bool any;          // a size outside the register plans (spo1d_any.cu)
    AnyPlan ap;
    double2* d_tw;     // its twiddle table
  };
  bool index_dirty = true;
  std::vector<Class> classes;
  // persistent launch: items of packets (one size class each), claimed by
  // the CTAs of one kernel in decreasing cost
  int launch = ESPEC_LAUNCH_CLASSES;
  bool persist_ok = false;           // every packet size has a persistent class
  std::vector<SpoItem> items;        // in claim order
  std::vector<int> slot_pk;          // packet index of each slot of the item list
  std::map<int, double> item_cost;   // per packet size: cost of one item
  SpoItem* d_items = nullptr;
  SpoPacket* d_pk_items = nullptr;   // packet descriptors in slot order
  unsigned int* d_next = nullptr;    // claim counter
  bool items_dirty = true;
  int items_steps = -1;              // nsteps the item descriptors' C(t) offsets are for
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  cudaEvent_t ev_fork = nullptr;
  // device buffers
  double* d_vpot = nullptr;
  double* d_vabc = nullptr;
  double2* d_psi0 = nullptr;
  double2* d_psi = nullptr;
  double* d_tc = nullptr;
  int* d_kperm = nullptr;
  int* d_pk_of = nullptr;
  int* d_pk_off = nullptr;
  double* d_kscale = nullptr;
  void* d_tab = nullptr;
  size_t tab_bytes = 0;
  double2* d_c = nullptr;
  int c_cap_steps = -1;  // nsteps the C(t) buffer was sized for
  double* d_kq_c = nullptr;
  double* d_kq_s = nullptr;
  bool loaded = false;
  bool has_prev = false;      // SOD: d_psi_prev holds psi(t - dt) of the current state
  double2* d_diag = nullptr;  // (E, norm) per packet
  int* d_nonfinite = nullptr; // packets whose C(t) went non-finite in the last run
  HostStage stage;            // host transfers: (re | im) blocks, contiguous
  // tables (sub-pointers of d_tab)
  SpoTables<double> t64{};
  SpoTables<float> t32{};
};

static void plan_free(espec_spo_plan* p) {
  for (auto& c : p->classes) {
    cudaFree(c.d_pk);
    if (c.d_pkd) cudaFree(c.d_pkd);
    if (c.d_kfreq) cudaFree(c.d_kfreq);
    if (c.d_tw) cudaFree(c.d_tw);
  }
  for (auto s : p->streams) cudaStreamDestroy(s);
  for (auto e : p->events) cudaEventDestroy(e);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  void* bufs[] = {p->d_vpot, p->d_vabc, p->d_psi0, p->d_psi,  p->d_tc,       p->d_kperm,
                  p->d_pk_of, p->d_pk_off, p->d_kscale, p->d_tab, p->d_c,  p->d_kq_c,
                  p->d_kq_s, p->d_psi_prev, p->d_diag, p->d_items, p->d_pk_items, p->d_next,
                  p->d_nonfinite};
  for (void* b : bufs)
    if (b) cudaFree(b);
  p->stage.release();
}

#define ESPEC_CK(call)                                           \
  do {                                                           \
    cudaError_t e_ = (call);                                     \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_);     \
  } while (0)

// host-built index tables: DIGT, final-position frequencies of the chosen
// plans, packet ids and kinetic scales
static int spo_index_tables(espec_spo_plan* p) {
  const size_t np = p->npts;
  const int npk = p->npk;
  int rc = 0;
  std::vector<double> tc(np), kscale(npk);
  std::vector<int> kperm(np), pk_of(np);
  std::map<int, int> var_of;
  const bool persist = p->launch == ESPEC_LAUNCH_PERSISTENT;
  // the reference-defect form always runs DefaultPlan<N> (launch_variant),
  // so its tables take that plan's final layout whatever the class's variant
  const bool quirk = p->method == ESPEC_SPO && (p->quirks & ESPEC_Q_SPO_INPLACE);
  for (auto& c : p->classes)
    var_of[c.n] = persist ? persist_variant(c.n, p->precision == ESPEC_FP64)
                          : (quirk ? 0 : c.variant);
  std::map<int, std::pair<std::vector<int>, int>> kap_cache;
  for (int i = 0; i < npk; ++i) {
    const int n = p->n[i];
    digt_1d(n, p->sh[i], p->sm[i], tc.data() + p->off[i]);
    auto it = kap_cache.find(n);
    if (it == kap_cache.end()) {
      std::vector<int> kap;
      int n3 = 0;
      plan_info(n, var_of[n], kap, n3);
      it = kap_cache.emplace(n, std::make_pair(kap, n3)).first;
    }
    for (int j = 0; j < n; ++j) {
      kperm[p->off[i] + j] = it->second.first[j];
      pk_of[p->off[i] + j] = i;
    }
    // round trip gain: N, divided by 3 per unitary radix-3 stage of the FP32 form
    double gain = n;
    if (p->precision == ESPEC_MIXED)
      for (int k = 0; k < it->second.second; ++k) gain /= 3.0;
    kscale[i] = 1.0 / gain;
  }
  if ((rc = ck(cudaMemcpy(p->d_tc, tc.data(), np * 8, cudaMemcpyHostToDevice), "H2D"))) return rc;
  if ((rc = ck(cudaMemcpy(p->d_kperm, kperm.data(), np * 4, cudaMemcpyHostToDevice), "H2D")))
    return rc;
  if ((rc = ck(cudaMemcpy(p->d_pk_of, pk_of.data(), np * 4, cudaMemcpyHostToDevice), "H2D")))
    return rc;
  if ((rc = ck(cudaMemcpy(p->d_pk_off, p->off.data(), npk * 4, cudaMemcpyHostToDevice), "H2D")))
    return rc;
  if ((rc = ck(cudaMemcpy(p->d_kscale, kscale.data(), npk * 8, cudaMemcpyHostToDevice), "H2D")))
    return rc;
  p->index_dirty = false;
  return ESPEC_OK;
}

extern "C" int espec_prop_create(espec_spo_plan** out, int npk, const int* npts,
                                 const double* sh, const double* sm, double dt_fs, int method,
                                 int precision, int absorb, int quirks) {
  if (!out || npk <= 0 || !npts || !sh || !sm) return set_error(ESPEC_EINVAL, "null argument");
  if (method != ESPEC_SPO && method != ESPEC_SOD)
    return set_error(ESPEC_EINVAL, "method must be ESPEC_SPO or ESPEC_SOD");
  if (method == ESPEC_SOD && precision != ESPEC_FP64)
    return set_error(ESPEC_EINVAL, "the SOD propagator runs in FP64 only");
  if (method == ESPEC_SOD && (quirks & ESPEC_Q_SPO_INPLACE))
    return set_error(ESPEC_EINVAL, "ESPEC_Q_SPO_INPLACE applies to the split-operator method");
  if (precision != ESPEC_FP64 && precision != ESPEC_MIXED)
    return set_error(ESPEC_EINVAL, "precision must be ESPEC_FP64 or ESPEC_MIXED");
  if (precision == ESPEC_MIXED && (quirks & ESPEC_Q_SPO_INPLACE))
    return set_error(ESPEC_EINVAL, "the reference-defect mode exists for FP64 only");
  if (absorb < ESPEC_ABS_NONE || absorb > ESPEC_ABS_SMOOTHW)
    return set_error(ESPEC_EINVAL, "unknown absorber type");
  auto* p = new espec_spo_plan;
  p->method = method;
  p->npk = npk;
  p->precision = precision;
  p->absorb = absorb;
  p->quirks = quirks;
  p->dt_fs = dt_fs;
  p->n.assign(npts, npts + npk);
  p->sh.assign(sh, sh + npk);
  p->sm.assign(sm, sm + npk);
  p->off.resize(npk + 1);
  p->off[0] = 0;
  // sizes outside the register plans run the any-size kernels (FP64)
  auto native = [&](int n) {
    return size_supported(n) && (method != ESPEC_SOD || sod_size_supported(n));
  };
  for (int i = 0; i < npk; ++i) {
    AnyPlan ap;
    if (!native(p->n[i]) && (precision != ESPEC_FP64 || !any_plan(p->n[i], ap) ||
                             any_smem_bytes(p->n[i], method) > kMaxSmem)) {
      delete p;
      return set_error(ESPEC_EINVAL, precision != ESPEC_FP64
                                         ? "unsupported packet size for the mixed form (256, 384, "
                                           "512, 768, 1024, 1536, 2048, 4096)"
                                         : "unsupported packet size (FP64: even sizes from 4 to "
                                           "7252 points, 3626 for SOD)");
    }
    if ((long long)p->off[i] + p->n[i] > INT_MAX) {
      delete p;
      return set_error(ESPEC_EINVAL, "more than 2^31 - 1 grid points in one plan");
    }
    p->off[i + 1] = p->off[i] + p->n[i];
  }
  p->npts = p->off[npk];
  int rc = 0;
  auto fail = [&](int code) {
    plan_free(p);
    delete p;
    return code;
  };
  // size classes, largest first so that the longest CTAs start first
  std::map<int, std::vector<SpoPacket>, std::greater<int>> cls;
  for (int i = 0; i < npk; ++i) cls[p->n[i]].push_back(SpoPacket{p->off[i], 0});
  for (auto& kv : cls) {
    espec_spo_plan::Class c{kv.first, (int)kv.second.size(), nullptr,
                            method == ESPEC_SOD ? 0 : default_variant(kv.first, precision),
                            nullptr, nullptr, !native(kv.first), AnyPlan{}, nullptr};
    p->classes.push_back(c);  // owned by the plan from here on (freed by plan_free)
    auto& cc = p->classes.back();
    if ((rc = ck(cudaMalloc(&cc.d_pk, sizeof(SpoPacket) * cc.count), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&cc.d_pkd, sizeof(SpoPacket) * cc.count), "cudaMalloc")))
      return fail(rc);
    if ((rc = ck(cudaMalloc(&cc.d_kfreq, sizeof(int) * cc.n), "cudaMalloc"))) return fail(rc);
    if (cc.any) {
      any_plan(cc.n, cc.ap);
      std::vector<double2> tw(cc.n);
      any_twiddles(cc.n, tw.data());
      if ((rc = ck(cudaMalloc(&cc.d_tw, sizeof(double2) * cc.n), "cudaMalloc"))) return fail(rc);
      if ((rc = ck(cudaMemcpy(cc.d_tw, tw.data(), sizeof(double2) * cc.n, cudaMemcpyHostToDevice),
                   "H2D")))
        return fail(rc);
    }
    {
      std::vector<SpoPacket> pkd;
      for (int i = 0; i < npk; ++i)
        if (p->n[i] == cc.n) pkd.push_back(SpoPacket{p->off[i], i});
      std::vector<int> kap;
      int n3 = 0;
      plan_info(cc.n, 0, kap, n3);
      if ((rc = ck(cudaMemcpy(cc.d_pkd, pkd.data(), sizeof(SpoPacket) * pkd.size(),
                              cudaMemcpyHostToDevice), "H2D")))
        return fail(rc);
      if ((rc = ck(cudaMemcpy(cc.d_kfreq, kap.data(), sizeof(int) * cc.n, cudaMemcpyHostToDevice),
                   "H2D")))
        return fail(rc);
    }
    cudaStream_t s;
    if ((rc = ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream"))) return fail(rc);
    p->streams.push_back(s);
    cudaEvent_t e;
    if ((rc = ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))) return fail(rc);
    p->events.push_back(e);
  }
  if ((rc = ck(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming), "event")))
    return fail(rc);
  const size_t np = p->npts;
  if ((rc = ck(cudaMalloc(&p->d_vpot, np * 8), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_vabc, np * 8), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_psi0, np * 16), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_psi, np * 16), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_tc, np * 8), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_kperm, np * 4), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_pk_of, np * 4), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_pk_off, npk * 4), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_kscale, npk * 8), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_diag, npk * 16), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMalloc(&p->d_nonfinite, sizeof(int)), "cudaMalloc"))) return fail(rc);
  if ((rc = ck(cudaMemset(p->d_nonfinite, 0, sizeof(int)), "cudaMemset"))) return fail(rc);
  if (precision == ESPEC_FP64) {
    p->tab_bytes = np * 16 * 5;
  } else {
    p->tab_bytes = np * (12 * 4 + 8);
  }
  if ((rc = ck(cudaMalloc(&p->d_tab, p->tab_bytes), "cudaMalloc"))) return fail(rc);
  if (method == ESPEC_SOD) {
    if ((rc = ck(cudaMalloc(&p->d_psi_prev, np * 16), "cudaMalloc"))) return fail(rc);
    double* tb = (double*)p->d_tab;  // 40 B per point inside the 80 B FP64 table block
    p->tsod.vc = tb;
    p->tsod.kc = tb + np;
    p->tsod.ab = tb + 2 * np;
    p->tsod.w = (const cpx<double>*)(tb + 3 * np);
  }
  if (quirks & ESPEC_Q_SPO_INPLACE) {
    if ((rc = ck(cudaMalloc(&p->d_kq_c, np * 8), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_kq_s, np * 8), "cudaMalloc"))) return fail(rc);
  }
  char* tb = (char*)p->d_tab;
  if (precision == ESPEC_FP64) {
    auto* c = (cpx<double>*)tb;
    p->t64.g = c;
    p->t64.h = c + np;
    p->t64.hm = c + 2 * np;
    p->t64.k = c + 3 * np;
    p->t64.w = c + 4 * np;
  } else {
    auto* c = (Tab<float>::phase_t*)tb;
    p->t32.g = c;
    p->t32.h = c + np;
    p->t32.hm = c + 2 * np;
    p->t32.k = c + 3 * np;
    p->t32.w = (cpx<float>*)(c + 4 * np);  // 12-byte phases: w stays 4-byte aligned
  }
  // the persistent launch covers the SPO method without the in-place defect
  // when every packet size has a class in the persistent kernel; it is an
  // option (espec_spo_set_launch): on the 4096-packet Morse scan one kernel
  // per size class with each size's own variant runs 6-9% faster
  p->persist_ok = method == ESPEC_SPO && !(quirks & ESPEC_Q_SPO_INPLACE);
  for (int i = 0; i < npk && p->persist_ok; ++i) p->persist_ok = persist_class(p->n[i]) >= 0;
  if (p->persist_ok) {
    if ((rc = ck(cudaMalloc(&p->d_pk_items, sizeof(SpoPacket) * npk), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_items, sizeof(SpoItem) * npk), "cudaMalloc"))) return fail(rc);
    if ((rc = ck(cudaMalloc(&p->d_next, sizeof(unsigned int)), "cudaMalloc"))) return fail(rc);
  }
  if ((rc = spo_index_tables(p))) return fail(rc);
  *out = p;
  return ESPEC_OK;
}

extern "C" int espec_spo_create(espec_spo_plan** out, int npk, const int* npts,
                                const double* sh, const double* sm, double dt_fs, int precision,
                                int absorb, int quirks) {
  return espec_prop_create(out, npk, npts, sh, sm, dt_fs, ESPEC_SPO, precision, absorb, quirks);
}

extern "C" int espec_spo_set_variant(espec_spo_plan* p, int npts, int variant) {
  if (!p) return set_error(ESPEC_EINVAL, "null plan");
  if (p->method != ESPEC_SPO) return set_error(ESPEC_EINVAL, "variants exist for ESPEC_SPO only");
  if (variant == ESPEC_VARIANT_TC) {
    if (npts != 256 || p->precision != ESPEC_MIXED)
      return set_error(ESPEC_EINVAL, "the tensor-core variant runs 256-point packets, mixed form");
  } else if (variant < 0 || variant >= kNumVariants) {
    return set_error(ESPEC_EINVAL, "unknown variant");
  } else if (!variant_fits(npts, variant, p->precision)) {
    return set_error(ESPEC_EINVAL, "variant needs more shared memory than a CTA can have");
  }
  bool found = false;
  for (auto& c : p->classes)
    if (c.n == npts) {
      if (c.any) return set_error(ESPEC_EINVAL, "packets of this size have one kernel (any size)");
      c.variant = variant;
      found = true;
    }
  if (!found) return set_error(ESPEC_EINVAL, "no packet of that size in the plan");
  p->launch = ESPEC_LAUNCH_CLASSES;  // the persistent kernel has fixed variants
  p->index_dirty = true;
  p->loaded = false;  // tables depend on the plan's final layout
  return ESPEC_OK;
}

extern "C" int espec_spo_set_launch(espec_spo_plan* p, int mode) {
  if (!p) return set_error(ESPEC_EINVAL, "null plan");
  if (mode != ESPEC_LAUNCH_CLASSES && mode != ESPEC_LAUNCH_PERSISTENT)
    return set_error(ESPEC_EINVAL, "unknown launch shape");
  if (mode == ESPEC_LAUNCH_PERSISTENT && !p->persist_ok)
    return set_error(ESPEC_EINVAL, "the persistent launch needs a split-operator plan without "
                                   "the in-place defect and packet sizes 256..2048");
  if (mode != p->launch) {
    p->launch = mode;
    p->index_dirty = true;
    p->loaded = false;  // the final layouts of the two shapes may differ
  }
  return ESPEC_OK;
}

extern "C" int espec_spo_set_item_cost(espec_spo_plan* p, int npts, double cost) {
  if (!p || !(cost > 0.0)) return set_error(ESPEC_EINVAL, "null plan or non-positive cost");
  p->item_cost[npts] = cost;
  p->items_dirty = true;
  return ESPEC_OK;
}

extern "C" int espec_spo_variant_count(void) { return kNumVariants; }

extern "C" void espec_spo_destroy(espec_spo_plan* p) {
  if (!p) return;
  plan_free(p);
  delete p;
}

extern "C" int espec_spo_npoints(const espec_spo_plan* p) { return p ? p->npts : -1; }

// set-up of all tables from state already in the plan's device buffers
static int spo_build_tables(espec_spo_plan* p, cudaStream_t st) {
  if (p->index_dirty) {
    int rc = spo_index_tables(p);
    if (rc) return rc;
  }
  SetupArgs a{};
  a.vpot = p->d_vpot;
  a.vabc = p->d_vabc;
  a.psi0 = p->d_psi0;
  a.tc = p->d_tc;
  a.kperm = p->d_kperm;
  a.pk_of = p->d_pk_of;
  a.pk_off = p->d_pk_off;
  a.kscale = p->d_kscale;
  a.npts = p->npts;
  a.cst1 = p->dt_fs / ESPEC_SHFS;
  a.cst2 = p->dt_fs / (2.0 * ESPEC_SHFS);
  a.absorb = p->absorb;
  a.fp32 = p->precision == ESPEC_MIXED;
  a.g64 = const_cast<cpx<double>*>(p->t64.g);
  a.h64 = const_cast<cpx<double>*>(p->t64.h);
  a.hm64 = const_cast<cpx<double>*>(p->t64.hm);
  a.k64 = const_cast<cpx<double>*>(p->t64.k);
  a.w64 = const_cast<cpx<double>*>(p->t64.w);
  a.g32 = const_cast<Tab<float>::phase_t*>(p->t32.g);
  a.h32 = const_cast<Tab<float>::phase_t*>(p->t32.h);
  a.hm32 = const_cast<Tab<float>::phase_t*>(p->t32.hm);
  a.k32 = const_cast<Tab<float>::phase_t*>(p->t32.k);
  a.w32 = const_cast<cpx<float>*>(p->t32.w);
  a.kq_c = p->d_kq_c;
  a.kq_s = p->d_kq_s;
  const int bs = 256;
  if (p->method == ESPEC_SOD) {
    sod_setup_kernel<<<(p->npts + bs - 1) / bs, bs, 0, st>>>(a, p->tsod, 2.0 * p->dt_fs / ESPEC_SHFS);
  } else {
    spo_setup_kernel<<<(p->npts + bs - 1) / bs, bs, 0, st>>>(a);
  }
  int rc = ck(cudaGetLastError(), "set-up kernel");
  if (rc) return rc;
  p->loaded = true;
  return ESPEC_OK;
}

extern "C" int espec_spo_load(espec_spo_plan* p, const double* vpot, const double* vabc,
                              const double* psi_re, const double* psi_im, int where,
                              void* stream) {
  if (!p || !vpot || !psi_re) return set_error(ESPEC_EINVAL, "null argument");
  if (p->absorb != ESPEC_ABS_NONE && !vabc) return set_error(ESPEC_EINVAL, "absorber table missing");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t np = p->npts;
  const cudaMemcpyKind kind = on_host(where) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  ESPEC_CK(cudaMemcpyAsync(p->d_vpot, vpot, np * 8, kind, st));
  if (vabc) ESPEC_CK(cudaMemcpyAsync(p->d_vabc, vabc, np * 8, kind, st));
  int rc = put_complex(p->stage, p->d_psi0, psi_re, psi_im, np, where, st);
  if (rc) return rc;
  // the current state of a freshly loaded plan is psi0
  ESPEC_CK(cudaMemcpyAsync(p->d_psi, p->d_psi0, np * 16, cudaMemcpyDeviceToDevice, st));
  p->has_prev = false;
  return spo_build_tables(p, st);
}

// Items of the persistent launch: the packets of each size in groups of
// persist_group(n) (one CTA's worth), ordered by decreasing cost of an item
// (longest processing time first; default cost = points of an item x log2 n),
// and their packet descriptors in slot order with the C(t) offsets of a run
// of nsteps steps.
static int persist_items(espec_spo_plan* p, int nsteps) {
  const bool d = p->precision == ESPEC_FP64;
  struct Raw {
    SpoItem it;
    double cost;
    std::vector<int> pk;
  };
  std::vector<Raw> raw;
  std::map<int, std::vector<int>> by_size;
  for (int i = 0; i < p->npk; ++i) by_size[p->n[i]].push_back(i);
  for (auto& kv : by_size) {
    const int n = kv.first, g = persist_group(n, d), cls = persist_class(n);
    if (g < 1 || cls < 0) return set_error(ESPEC_EINVAL, "packet size without a persistent class");
    auto c = p->item_cost.find(n);
    const double cost = c != p->item_cost.end() ? c->second : (double)g * n * std::log2((double)n);
    for (size_t k = 0; k < kv.second.size(); k += g) {
      Raw r;
      r.it.cls = cls;
      r.it.count = (int)std::min<size_t>(g, kv.second.size() - k);
      r.it.first = 0;
      r.cost = cost;
      r.pk.assign(kv.second.begin() + k, kv.second.begin() + k + r.it.count);
      raw.push_back(std::move(r));
    }
  }
  std::stable_sort(raw.begin(), raw.end(), [](const Raw& a, const Raw& b) { return a.cost > b.cost; });
  p->items.clear();
  p->slot_pk.clear();
  std::vector<SpoPacket> pk;
  for (auto& r : raw) {
    r.it.first = (int)p->slot_pk.size();
    p->items.push_back(r.it);
    for (int i : r.pk) {
      p->slot_pk.push_back(i);
      pk.push_back(SpoPacket{p->off[i], (long long)i * (nsteps + 1)});
    }
  }
  ESPEC_CK(cudaMemcpy(p->d_items, p->items.data(), sizeof(SpoItem) * p->items.size(),
                      cudaMemcpyHostToDevice));
  ESPEC_CK(cudaMemcpy(p->d_pk_items, pk.data(), sizeof(SpoPacket) * pk.size(),
                      cudaMemcpyHostToDevice));
  p->items_dirty = false;
  return ESPEC_OK;
}

// the whole batch in one persistent launch
static int persist_launch(espec_spo_plan* p, int nsteps, bool resume, cudaStream_t st) {
  ESPEC_CK(cudaMemsetAsync(p->d_next, 0, sizeof(unsigned int), st));
  cudaError_t e;
  if (p->precision == ESPEC_FP64) {
    SpoPersistArgs<double> pa{};
    pa.a.tab = p->t64;
    pa.a.pk = p->d_pk_items;
    pa.a.psi0 = p->d_psi0;
    if (resume) pa.a.psi_start = p->d_psi;
    pa.a.psi_out = p->d_psi;
    pa.a.c_out = p->d_c;
    pa.a.nsteps = nsteps;
    pa.a.nonfinite = p->d_nonfinite;
    pa.items = p->d_items;
    pa.nitems = (int)p->items.size();
    pa.next = p->d_next;
    e = spo_persist_launch_f64(pa, st);
  } else {
    SpoPersistArgs<float> pa{};
    pa.a.tab = p->t32;
    pa.a.pk = p->d_pk_items;
    pa.a.psi0 = p->d_psi0;
    if (resume) pa.a.psi_start = p->d_psi;
    pa.a.psi_out = p->d_psi;
    pa.a.c_out = p->d_c;
    pa.a.nsteps = nsteps;
    pa.a.nonfinite = p->d_nonfinite;
    pa.items = p->d_items;
    pa.nitems = (int)p->items.size();
    pa.next = p->d_next;
    e = spo_persist_launch_f32(pa, st);
  }
  if (e != cudaSuccess) return set_cuda_error("spo1d_persistent launch", e);
  return ESPEC_OK;
}

// one launch per size class over nsteps steps, from psi0 (resume = false) or
// from the plan's current state (resume = true)
static int prop_launch(espec_spo_plan* p, int nsteps, bool resume, cudaStream_t st) {
  if (p->c_cap_steps != nsteps) {
    if (p->d_c) cudaFree(p->d_c);
    p->d_c = nullptr;
    ESPEC_CK(cudaMalloc(&p->d_c, sizeof(double2) * (size_t)p->npk * (nsteps + 1)));
    p->c_cap_steps = nsteps;
    // packet descriptors carry the C(t) offsets
    std::map<int, std::vector<SpoPacket>> cls;
    for (int i = 0; i < p->npk; ++i)
      cls[p->n[i]].push_back(SpoPacket{p->off[i], (long long)i * (nsteps + 1)});
    for (auto& c : p->classes) {
      auto& v = cls[c.n];
      ESPEC_CK(cudaMemcpy(c.d_pk, v.data(), sizeof(SpoPacket) * v.size(), cudaMemcpyHostToDevice));
    }
  }
  const bool quirk = (p->quirks & ESPEC_Q_SPO_INPLACE) != 0;
  ESPEC_CK(cudaMemsetAsync(p->d_nonfinite, 0, sizeof(int), st));
  if (p->method == ESPEC_SPO && p->launch == ESPEC_LAUNCH_PERSISTENT) {
    if (p->items_dirty || p->items_steps != nsteps) {
      int rc = persist_items(p, nsteps);
      if (rc) return rc;
      p->items_steps = nsteps;
    }
    return persist_launch(p, nsteps, resume, st);
  }
  ESPEC_CK(cudaEventRecord(p->ev_fork, st));
  for (size_t ci = 0; ci < p->classes.size(); ++ci) {
    auto& c = p->classes[ci];
    cudaStream_t cs = p->streams[ci];
    ESPEC_CK(cudaStreamWaitEvent(cs, p->ev_fork, 0));
    cudaError_t e;
    if (p->method == ESPEC_SOD) {
      SodArgs a{};
      a.tab = p->tsod;
      a.pk = c.d_pk;
      a.psi0 = p->d_psi0;
      if (resume) {
        a.psi_start = p->d_psi;
        a.psi_prev_start = p->d_psi_prev;
      }
      a.psi_out = p->d_psi;
      a.psi_prev_out = p->d_psi_prev;
      a.c_out = p->d_c;
      a.nsteps = nsteps;
      int kabs = p->absorb == ESPEC_ABS_VOPTIC ? 1 : (p->absorb == ESPEC_ABS_SMOOTHW ? 2 : 0);
      if (kabs == 2 && (p->quirks & ESPEC_Q_SOD_SMOOTHW)) kabs = 0;  // sodfft.f:108
      e = c.any ? sod_any_launch(a, c.ap, c.d_tw, kabs, c.count, cs)
                : sod_launch(c.n, kabs, a, c.count, cs);
    } else if (p->precision == ESPEC_FP64) {
      SpoArgs<double> a{};
      a.tab = p->t64;
      a.pk = c.d_pk;
      a.psi0 = p->d_psi0;
      if (resume) a.psi_start = p->d_psi;
      a.psi_out = p->d_psi;
      a.c_out = p->d_c;
      a.kq_c = p->d_kq_c;
      a.kq_s = p->d_kq_s;
      a.kq_scale = 1.0 / c.n;
      a.nsteps = nsteps;
      a.nonfinite = p->d_nonfinite;
      e = c.any ? spo_any_launch(a, c.ap, c.d_tw, quirk, c.count, cs)
                : launch_n<double>(c.n, c.variant, a, c.count, quirk, cs);
    } else {
      SpoArgs<float> a{};
      a.tab = p->t32;
      a.pk = c.d_pk;
      a.psi0 = p->d_psi0;
      if (resume) a.psi_start = p->d_psi;
      a.psi_out = p->d_psi;
      a.c_out = p->d_c;
      a.nsteps = nsteps;
      a.nonfinite = p->d_nonfinite;
      e = c.variant == ESPEC_VARIANT_TC ? spo_tc256_launch(a, c.count, cs)
                                         : launch_n<float>(c.n, c.variant, a, c.count, false, cs);
    }
    if (e != cudaSuccess) return set_cuda_error("spo1d_kernel launch", e);
    ESPEC_CK(cudaEventRecord(p->events[ci], cs));
    ESPEC_CK(cudaStreamWaitEvent(st, p->events[ci], 0));
  }
  if (p->method == ESPEC_SOD) p->has_prev = true;
  return ESPEC_OK;
}

extern "C" int espec_spo_run(espec_spo_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_spo_load has not been called");
  return prop_launch(p, nsteps, false, (cudaStream_t)stream);
}

extern "C" int espec_prop_continue(espec_spo_plan* p, int nsteps, void* stream) {
  if (!p || nsteps < 0) return set_error(ESPEC_EINVAL, "bad plan or step count");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_spo_load has not been called");
  if (p->method == ESPEC_SOD && !p->has_prev)
    return set_error(ESPEC_EINVAL, "a SOD plan continues a run: call espec_spo_run first");
  return prop_launch(p, nsteps, true, (cudaStream_t)stream);
}

extern "C" int espec_prop_energies(espec_spo_plan* p, double* e, double* norm, void* stream) {
  if (!p || !e || !norm) return set_error(ESPEC_EINVAL, "null argument");
  if (!p->loaded) return set_error(ESPEC_EINVAL, "espec_spo_load has not been called");
  cudaStream_t st = (cudaStream_t)stream;
  for (auto& c : p->classes) {
    DiagArgs a{p->d_psi, p->d_vpot, p->d_tc, c.d_kfreq, c.d_pkd, p->d_diag};
    cudaError_t err = c.any ? diag_any_launch(a, c.ap, c.d_tw, c.count, st)
                            : diag_launch(c.n, a, c.count, st);
    if (err != cudaSuccess) return set_cuda_error("diag1d_kernel launch", err);
  }
  std::vector<double2> h(p->npk);
  ESPEC_CK(cudaMemcpyAsync(h.data(), p->d_diag, 16 * (size_t)p->npk, cudaMemcpyDeviceToHost, st));
  ESPEC_CK(cudaStreamSynchronize(st));
  for (int i = 0; i < p->npk; ++i) {
    e[i] = h[i].x;
    norm[i] = h[i].y;
  }
  return ESPEC_OK;
}

extern "C" int espec_spo_results(espec_spo_plan* p, double* c_re, double* c_im, double* psi_re,
                                 double* psi_im, int where, void* stream) {
  if (!p || p->c_cap_steps < 0) return set_error(ESPEC_EINVAL, "no results: run the plan first");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t nc = (size_t)p->npk * (p->c_cap_steps + 1);
  int rc = get_complex(p->stage, p->d_c, c_re, c_im, nc, where, st);
  if (rc == ESPEC_OK) rc = get_complex(p->stage, p->d_psi, psi_re, psi_im, p->npts, where, st);
  if (rc) return rc;
  if (where == ESPEC_MEM_HOST) ESPEC_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}

extern "C" const void* espec_spo_device_c(const espec_spo_plan* p) { return p ? p->d_c : nullptr; }

extern "C" int espec_spo_tc_status(int* timed_out) {
  if (!timed_out) return set_error(ESPEC_EINVAL, "null argument");
  return spo_tc_status(timed_out);
}

extern "C" int espec_prop_nonfinite(espec_spo_plan* p, int* count, void* stream) {
  if (!p || !count) return set_error(ESPEC_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  ESPEC_CK(cudaMemcpyAsync(count, p->d_nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st));
  ESPEC_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}

extern "C" int espec_prop_previous(espec_spo_plan* p, double* psi_re, double* psi_im, int where,
                                   void* stream) {
  if (!p || p->method != ESPEC_SOD || p->c_cap_steps < 0)
    return set_error(ESPEC_EINVAL, "previous state exists for run SOD plans only");
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = get_complex(p->stage, p->d_psi_prev, psi_re, psi_im, p->npts, where, st);
  if (rc) return rc;
  if (where == ESPEC_MEM_HOST) ESPEC_CK(cudaStreamSynchronize(st));
  return ESPEC_OK;
}
