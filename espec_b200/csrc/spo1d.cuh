// spo1d.cuh -- persistent batched 1D split-operator propagation (device side).
//
// One CTA owns one packet for the whole time loop; the wave function never
// leaves registers/shared memory between steps.  Per step (Strang splitting
// with the two V half-steps of consecutive steps merged, spofft.f:120-191):
//
//   phi <- g . phi            x space, g = e^{-i V dt} (x absorber)   [h at step 1]
//   phi <- F^-1 K F phi       K = e^{-i T(k) dt} / N  (k space)
//   C(t) = sum_j w_j phi_j    w = conj(psi0) . h      (FP64 accumulation)
//
// psi(t) = h . phi (x mask) is formed only once at the end.  The forward FFT
// is a decimation-in-frequency Stockham sequence whose output stays in the
// registers of the thread that computed the last butterflies; the inverse
// runs the exact conjugate stages in reverse order, so each step needs
// 2(S-1) shared-memory exchanges for S radix stages and no transposes.  The
// half-swaps of spofft.f:120-133/178-191 (an fftshift before the forward and
// after the inverse transform) cancel exactly and are not performed.
#pragma once
#include <string.h>

#include "cplx.cuh"

namespace espec {

// ---------------------------------------------------------------------------
// radix plans: P points per thread, radices in execution order
// ---------------------------------------------------------------------------
template <int N_, int P_, int... Rs>
struct Plan {
  static constexpr int N = N_;
  static constexpr int P = P_;
  static constexpr int T = N_ / P_;
  static constexpr int S = sizeof...(Rs);
  static constexpr int r[S] = {Rs...};
  static __host__ __device__ constexpr int M(int s) {
    int m = N_;
    for (int i = 0; i < s; ++i) m /= r[i];
    return m;
  }
  // number of non-trivial twiddles held per thread (stages with M/R > 1)
  static __host__ __device__ constexpr int tw_off(int s) {
    int o = 0;
    for (int i = 0; i < s; ++i)
      if (M(i) / r[i] > 1) o += (P / r[i]) * (r[i] - 1);
    return o;
  }
  static constexpr int NTW = tw_off(S) > 0 ? tw_off(S) : 1;
  static __host__ __device__ constexpr int m(int s) { return M(s) / r[s]; }
  static __host__ __device__ constexpr int Q(int s) { return P_ / r[s]; }
  // butterflies of a warp form whole sub-problems at stage s
  static __host__ __device__ constexpr bool warp_aligned(int s) { return (32 * Q(s)) % m(s) == 0; }
  // the exchange between stages s and s+1 stays inside each warp
  static __host__ __device__ constexpr bool local(int s) {
    return T <= 32 || (warp_aligned(s) && warp_aligned(s + 1));
  }
  static __host__ __device__ constexpr int n_local() {
    int c = 0;
    for (int i = 0; i + 1 < S; ++i) c += local(i) ? 1 : 0;
    return c;
  }
  static __host__ __device__ constexpr int n_global() { return (S - 1) - n_local(); }
  // Shared buffers: CTA-wide exchanges alternate between buffers 0 and 1,
  // warp-local exchanges between buffers 2 and 3 (each kind alternates over
  // the forward then the inverse sequence; both counts per step are even).
  static __host__ __device__ constexpr int buf_fwd(int s) {
    int c = 0;
    for (int i = 0; i < s; ++i) c += (local(i) == local(s)) ? 1 : 0;
    return (local(s) ? 2 : 0) + (c & 1);
  }
  static __host__ __device__ constexpr int buf_inv(int s) {
    int c = local(s) ? n_local() : n_global();
    for (int i = S - 2; i > s; --i) c += (local(i) == local(s)) ? 1 : 0;
    return (local(s) ? 2 : 0) + (c & 1);
  }
  static constexpr int NBUF = (n_local() > 0 && n_global() > 0) ? 4 : 2;
  static constexpr bool valid() {
    int prod = 1;
    for (int i = 0; i < S; ++i) {
      if (P_ % r[i] != 0) return false;
      prod *= r[i];
    }
    return prod == N_ && N_ % P_ == 0;
  }
  static_assert(valid(), "radices must multiply to N and divide P");
  // number of unitary radix-3 factors (FP32 form keeps them unitary)
  static __host__ __device__ constexpr int n3() {
    int c = 0;
    for (int i = 0; i < S; ++i)
      if (r[i] % 3 == 0) ++c;
    return c;
  }

  // Shared-memory layout of exchange s (outputs of stage s -> inputs of
  // stage s+1): one of three XOR swizzles of the low four index bits, each a
  // bijection inside every 16-element block, chosen at compile time as the
  // one with the fewest bank conflicts for the exchange's store and load
  // patterns: 16-byte elements are served per quarter warp (8 lanes must hit
  // distinct index residues mod 8), 8-byte elements per half warp (16 lanes,
  // residues mod 16).  The radix-12 and radix-4 chains conflict under the
  // first swizzle (a stride-2 index pattern in their last exchanges).
  static __host__ __device__ constexpr int swz_apply(int kind, int i) {
    return kind == 0 ? i ^ (((i >> 3) ^ (i >> 4)) & 15)
                     : (kind == 1 ? i ^ (((i >> 1) ^ (i >> 2)) & 15) : i ^ (((i >> 1) ^ (i >> 3)) & 15));
  }
  static __host__ __device__ constexpr int c_beta(int s, int t, int q) {
    return (t >> 5) * 32 * Q(s) + (t & 31) + 32 * q;
  }
  // element of lane t: output k of butterfly q of stage s (out = true), or
  // input k of butterfly q of stage s
  static __host__ __device__ constexpr int c_pos(bool out, int s, int t, int q, int k) {
    const int m = M(s) / r[s], b = c_beta(s, t, q);
    return out ? ((b / m) * r[s] + k) * m + b % m : (b / m) * M(s) + b % m + m * k;
  }
  // extra wavefronts of one warp instruction of warp w, for elements of 16
  // and of 8 bytes
  static __host__ __device__ constexpr int extra(int kind, int w, bool out, int s, int q, int k) {
    int tot = 0;
    for (int es = 0; es < 2; ++es) {
      const int lanes = es == 0 ? 8 : 16;
      for (int g = 0; g < 32; g += lanes) {
        int cnt[16] = {}, mx = 0;
        for (int l = g; l < g + lanes && w * 32 + l < T; ++l) {
          const int res = swz_apply(kind, c_pos(out, s, w * 32 + l, q, k)) % lanes;
          cnt[res] += 1;
          if (cnt[res] > mx) mx = cnt[res];
        }
        if (mx > 1) tot += mx - 1;
      }
    }
    return tot;
  }
  static __host__ __device__ constexpr int conflicts(int s, int kind) {
    int tot = 0;
    const int W = T < 32 ? 1 : T / 32;
    for (int w = 0; w < W; ++w) {
      for (int q = 0; q < Q(s); ++q)
        for (int k = 0; k < r[s]; ++k) tot += extra(kind, w, true, s, q, k);
      for (int q = 0; q < Q(s + 1); ++q)
        for (int k = 0; k < r[s + 1]; ++k) tot += extra(kind, w, false, s + 1, q, k);
    }
    return tot;
  }
  static __host__ __device__ constexpr int swz_pick(int s) {
    int best = 0, bc = conflicts(s, 0);
    for (int kind = 1; kind < 3; ++kind) {
      const int c = conflicts(s, kind);
      if (c < bc) {
        best = kind;
        bc = c;
      }
    }
    return best;
  }
};

template <int N>
struct DefaultPlan;
// Default plans: one cross-warp stage first, then stages whose sub-problems
// fit inside one warp (32 * P points), so that only one exchange per
// transform needs a CTA-wide barrier and the others a warp barrier.
template <> struct DefaultPlan<256>  { using type = Plan<256, 8, 8, 8, 4>; };
template <> struct DefaultPlan<512>  { using type = Plan<512, 8, 2, 8, 8, 4>; };
template <> struct DefaultPlan<1024> { using type = Plan<1024, 8, 4, 8, 8, 4>; };
template <> struct DefaultPlan<2048> { using type = Plan<2048, 8, 8, 8, 8, 4>; };
template <> struct DefaultPlan<4096> { using type = Plan<4096, 16, 8, 16, 16, 2>; };
template <> struct DefaultPlan<384>  { using type = Plan<384, 12, 12, 4, 4, 2>; };
template <> struct DefaultPlan<768>  { using type = Plan<768, 12, 2, 12, 4, 4, 2>; };
template <> struct DefaultPlan<1536> { using type = Plan<1536, 12, 4, 12, 4, 4, 2>; };

// ---------------------------------------------------------------------------
// per-precision table formats
// ---------------------------------------------------------------------------
template <typename R>
struct Tab;
template <>
struct Tab<double> {
  using rot_t = RotD;
  using phase_t = cpx<double>;   // complex factor (rotation x magnitude)
  using weight_t = cpx<double>;
  static ESPEC_HD cpx<double> apply(const phase_t& f, cpx<double> a) {
    return mk(fma(a.x, f.x, -a.y * f.y), fma(a.x, f.y, a.y * f.x));
  }
};
template <>
struct Tab<float> {
  using rot_t = RotF;
  // lifting rotation by phi' followed by the real factor ag = g * a (the
  // exact negation of make_rotf folded into the magnitude a)
  struct phase_t {
    float t, s, ag;
  };
  using weight_t = cpx<float>;
  static ESPEC_HD cpx<float> apply(const phase_t& f, cpx<float> v) {
    float x = v.x, y = v.y;
    x = fmaf(-f.t, y, x);
    y = fmaf(f.s, x, y);
    x = fmaf(-f.t, y, x);
    return mk(x * f.ag, y * f.ag);
  }
};

// pointers of one precision's tables (all per point, concatenated over packets)
template <typename R>
struct SpoTables {
  const typename Tab<R>::phase_t* g;   // e^{-iV dt} (x absorber), x order
  const typename Tab<R>::phase_t* h;   // e^{-iV dt/2}, x order (first step)
  const typename Tab<R>::phase_t* hm;  // mask x e^{-iV dt/2}, x order (final psi)
  const typename Tab<R>::phase_t* k;   // kinetic phase x scale, final FFT layout
  const typename Tab<R>::weight_t* w;  // conj(psi0) x h (x mask), x order
};

struct SpoPacket {
  int off;         // first point of the packet in the concatenated arrays
  long long c_off;  // first C(t) sample of the packet (npk * (nsteps + 1) may pass 2^31)
};

template <typename R>
struct SpoArgs {
  SpoTables<R> tab;
  const SpoPacket* pk;      // per CTA (packets of this size class)
  const double2* psi0;      // initial psi (x order), FP64
  const double2* psi_start; // resume from this psi instead of psi0 (C(0) not written)
  double2* psi_out;         // psi(TF) (x order), FP64
  double2* c_out;           // C(t) samples, nsteps+1 per packet
  const double* kq_c;       // FP64 quirk form: cos(CST1*TC) per point (final layout)
  const double* kq_s;       //                    sin(CST1*TC)
  double kq_scale;          //                    1/N
  int nsteps;
  int* nonfinite;           // count of packets with a non-finite C(t) sample (or null)
};

// Sum of the NW per-warp partials of one C(t) sample, compensated
// (Neumaier: the rounding error of every addition is carried along and added
// back at the end), in warp order on one thread.
template <int NW>
__device__ __forceinline__ double2 sum_partials(const double2* cp) {
  double sr = 0.0, si = 0.0, er = 0.0, ei = 0.0;
#pragma unroll
  for (int i = 0; i < NW; ++i) {
    const double xr = cp[i].x, xi = cp[i].y;
    const double tr = sr + xr, ti = si + xi;
    er += fabs(sr) >= fabs(xr) ? (sr - tr) + xr : (xr - tr) + sr;
    ei += fabs(si) >= fabs(xi) ? (si - ti) + xi : (xi - ti) + si;
    sr = tr;
    si = ti;
  }
  return make_double2(sr + er, si + ei);
}

// Barrier of the T threads that propagate one packet.  A CTA may hold
// several such groups (the persistent kernel packs small packets): group g
// uses hardware barrier id g + 1 with T threads, a group that is the whole
// CTA uses id 0 (then bar.sync 0, T is __syncthreads).
template <int T>
__device__ __forceinline__ void group_bar(int id) {
  if constexpr (T <= 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(T) : "memory");
  }
}
template <int T>
__device__ __forceinline__ void group_sync() {
  group_bar<T>(0);
}

template <typename R, class PL>
struct SpoThread {
  static constexpr int N = PL::N, P = PL::P, T = PL::T, S = PL::S;
  using rot_t = typename Tab<R>::rot_t;
  // Warp-local exchanges need four buffers; when those would not fit next to
  // the tables every exchange uses a CTA-wide barrier and two buffers.
  static constexpr bool kLocal = PL::NBUF == 2 || (size_t)4 * N * sizeof(cpx<R>) <= 160 * 1024;
  static constexpr int NBUF = kLocal ? PL::NBUF : 2;
  template <int s>
  static __host__ __device__ constexpr bool local_x() {
    return kLocal ? PL::local(s) : (T <= 32);
  }
  template <int s>
  static __host__ __device__ constexpr int buf_f() {
    return kLocal ? (NBUF == 4 ? PL::buf_fwd(s) : (PL::buf_fwd(s) & 1)) : (s & 1);
  }
  template <int s>
  static __host__ __device__ constexpr int buf_i() {
    return kLocal ? (NBUF == 4 ? PL::buf_inv(s) : (PL::buf_inv(s) & 1)) : ((s + 1) & 1);
  }

  rot_t tw[PL::NTW];
  int bar = 0;  // hardware barrier id of this thread's packet group (group_bar)

  // shared-memory layout of exchange s (Plan::swz_pick, chosen at compile time)
  template <int s>
  static ESPEC_HD int sidx(int i) {
    constexpr int kind = PL::swz_pick(s);
    return PL::swz_apply(kind, i);
  }

  ESPEC_HD void init_twiddles(int t) { init_stage<0>(t); }

  // butterfly handled by thread t in slot q of stage s: warp-major, lanes
  // cyclic inside the warp (consecutive lanes -> consecutive butterflies)
  template <int s>
  static ESPEC_HD int beta(int t, int q) {
    constexpr int Q = PL::Q(s);
    return (t >> 5) * 32 * Q + (t & 31) + 32 * q;
  }

  template <int s>
  ESPEC_HD void init_stage(int t) {
    if constexpr (s < S) {
      constexpr int RR = PL::r[s];
      constexpr int M = PL::M(s);
      constexpr int m = M / RR;
      constexpr int Q = P / RR;
      if constexpr (m > 1) {
        constexpr int o = PL::tw_off(s);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int n1 = beta<s>(t, q) % m;
#pragma unroll
          for (int k = 1; k < RR; ++k) {
            int j = (n1 * k) % M;
            if (2 * j > M) j -= M;  // angle 2 pi j / M in (-pi, pi]
            const double phi = 6.283185307179586476925287 * (double)j / (double)M;
            if constexpr (sizeof(R) == 8) {
              RotD r;
#ifdef __CUDA_ARCH__
              sincospi(2.0 * (double)j / (double)M, &r.s, &r.c);
#else
              r.s = sin(phi);
              r.c = cos(phi);
#endif
              tw[o + q * (RR - 1) + k - 1] = r;
            } else {
              tw[o + q * (RR - 1) + k - 1] = make_rotf(phi);
            }
          }
        }
      }
      init_stage<s + 1>(t);
    }
  }

  // forward stage s: butterflies then twiddles (DIF)
  template <int s>
  ESPEC_HD void fwd_bfly(cpx<R>* v) const {
    constexpr int RR = PL::r[s];
    constexpr int m = PL::M(s) / RR;
    constexpr int Q = P / RR;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      dft<R, RR, false>(v + q * RR);
      if constexpr (m > 1) {
        constexpr int o = PL::tw_off(s);
#pragma unroll
        for (int k = 1; k < RR; ++k)
          v[q * RR + k] = rot<false>(tw[o + q * (RR - 1) + k - 1], v[q * RR + k]);
      }
    }
  }

  // inverse of stage s: conjugate twiddles then conjugate butterflies (DIT)
  template <int s>
  ESPEC_HD void inv_bfly(cpx<R>* v) const {
    constexpr int RR = PL::r[s];
    constexpr int m = PL::M(s) / RR;
    constexpr int Q = P / RR;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if constexpr (m > 1) {
        constexpr int o = PL::tw_off(s);
#pragma unroll
        for (int k = 1; k < RR; ++k)
          v[q * RR + k] = rot<true>(tw[o + q * (RR - 1) + k - 1], v[q * RR + k]);
      }
      dft<R, RR, true>(v + q * RR);
    }
  }

  // positions of stage-s outputs held by thread t (slot q*R + k')
  template <int s>
  static ESPEC_HD int out_pos(int t, int q, int k) {
    constexpr int RR = PL::r[s];
    constexpr int m = PL::M(s) / RR;
    const int b = beta<s>(t, q);
    const int p = b / m, n1 = b % m;
    return (p * RR + k) * m + n1;
  }
  // positions of stage-s inputs held by thread t (slot q*R + k)
  template <int s>
  static ESPEC_HD int in_pos(int t, int q, int k) {
    constexpr int RR = PL::r[s];
    constexpr int M = PL::M(s);
    constexpr int m = M / RR;
    const int b = beta<s>(t, q);
    const int p = b / m, n1 = b % m;
    return p * M + n1 + m * k;
  }

  template <int s>
  __device__ __forceinline__ void xsync() const {
    if constexpr (local_x<s>()) {
      __syncwarp();
    } else {
      group_bar<T>(bar);
    }
  }

  // exchange after forward stage s (s < S-1): outputs of s -> inputs of s+1
  template <int s>
  __device__ __forceinline__ void xchg_fwd(cpx<R>* v, cpx<R>* buf, int t) const {
    constexpr int R0 = PL::r[s], Q0 = P / R0;
    constexpr int R1 = PL::r[s + 1], Q1 = P / R1;
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int k = 0; k < R0; ++k) buf[sidx<s>(out_pos<s>(t, q, k))] = v[q * R0 + k];
    xsync<s>();
#pragma unroll
    for (int q = 0; q < Q1; ++q)
#pragma unroll
      for (int k = 0; k < R1; ++k) v[q * R1 + k] = buf[sidx<s>(in_pos<s + 1>(t, q, k))];
  }
  // reverse exchange: inputs of s+1 -> outputs of s
  template <int s>
  __device__ __forceinline__ void xchg_inv(cpx<R>* v, cpx<R>* buf, int t) const {
    constexpr int R0 = PL::r[s], Q0 = P / R0;
    constexpr int R1 = PL::r[s + 1], Q1 = P / R1;
#pragma unroll
    for (int q = 0; q < Q1; ++q)
#pragma unroll
      for (int k = 0; k < R1; ++k) buf[sidx<s>(in_pos<s + 1>(t, q, k))] = v[q * R1 + k];
    xsync<s>();
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int k = 0; k < R0; ++k) v[q * R0 + k] = buf[sidx<s>(out_pos<s>(t, q, k))];
  }

  template <int s>
  __device__ __forceinline__ void forward(cpx<R>* v, cpx<R>* bufs, int t) const {
    if constexpr (s < S) {
      fwd_bfly<s>(v);
      if constexpr (s + 1 < S) {
        xchg_fwd<s>(v, bufs + buf_f<s>() * N, t);
        forward<s + 1>(v, bufs, t);
      }
    }
  }
  template <int s>
  __device__ __forceinline__ void inverse(cpx<R>* v, cpx<R>* bufs, int t) const {
    if constexpr (s >= 0) {
      inv_bfly<s>(v);
      if constexpr (s > 0) {
        xchg_inv<s - 1>(v, bufs + buf_i<s - 1>() * N, t);
        inverse<s - 1>(v, bufs, t);
      }
    }
  }

  // x position held in slot j at the start/end of a step (stage-0 inputs)
  static ESPEC_HD int x_pos(int t, int j) {
    constexpr int R0 = PL::r[0];
    return in_pos<0>(t, j / R0, j % R0);
  }

  // final-layout position of slot j (for the k-space table)
  static ESPEC_HD int final_pos(int t, int j) {
    constexpr int RR = PL::r[S - 1];
    return out_pos<S - 1>(t, j / RR, j % RR);
  }
};

// ---------------------------------------------------------------------------
// where the per-point tables live during the time loop
//   kTab = 0: registers (P phases g, P kinetic phases k, P weights w per thread)
//   kTab = 1: shared memory, structure of arrays [component][slot][thread]
//            (conflict-free: consecutive threads read consecutive words)
// ---------------------------------------------------------------------------
template <typename R, class PL, int kTab>
struct TabStore;

template <typename R, class PL>
struct TabStore<R, PL, 0> {
  using ph = typename Tab<R>::phase_t;
  using wt = typename Tab<R>::weight_t;
  static constexpr size_t smem_bytes = 0;
  ph g[PL::P], k[PL::P];
  wt w[PL::P];
  __device__ __forceinline__ void init(void*) {}
  __device__ __forceinline__ void put(int j, int, const ph& gg, const ph& kk, const wt& ww) {
    g[j] = gg;
    k[j] = kk;
    w[j] = ww;
  }
  __device__ __forceinline__ ph G(int j, int) const { return g[j]; }
  __device__ __forceinline__ ph K(int j, int) const { return k[j]; }
  __device__ __forceinline__ wt W(int j, int) const { return w[j]; }
};

template <typename R, class PL>
struct TabStore<R, PL, 1> {
  using ph = typename Tab<R>::phase_t;
  using wt = typename Tab<R>::weight_t;
  static constexpr int CP = sizeof(ph) / sizeof(R);  // scalars per phase
  static constexpr int CW = sizeof(wt) / sizeof(R);
  static constexpr int P = PL::P, T = PL::T;
  static constexpr size_t smem_bytes = (size_t)(2 * CP + CW) * PL::N * sizeof(R);
  R* base;
  __device__ __forceinline__ void init(void* p) { base = reinterpret_cast<R*>(p); }
  template <typename X, int C>
  __device__ __forceinline__ void st(R* arr, int j, int t, const X& x) {
    R tmp[C];
    memcpy(tmp, &x, sizeof(X));
#pragma unroll
    for (int c = 0; c < C; ++c) arr[(c * P + j) * T + t] = tmp[c];
  }
  template <typename X, int C>
  __device__ __forceinline__ X ld(const R* arr, int j, int t) const {
    R tmp[C];
#pragma unroll
    for (int c = 0; c < C; ++c) tmp[c] = arr[(c * P + j) * T + t];
    X x;
    memcpy(&x, tmp, sizeof(X));
    return x;
  }
  __device__ __forceinline__ void put(int j, int t, const ph& gg, const ph& kk, const wt& ww) {
    st<ph, CP>(base, j, t, gg);
    st<ph, CP>(base + CP * PL::N, j, t, kk);
    st<wt, CW>(base + 2 * CP * PL::N, j, t, ww);
  }
  __device__ __forceinline__ ph G(int j, int t) const { return ld<ph, CP>(base, j, t); }
  __device__ __forceinline__ ph K(int j, int t) const { return ld<ph, CP>(base + CP * PL::N, j, t); }
  __device__ __forceinline__ wt W(int j, int t) const {
    return ld<wt, CW>(base + 2 * CP * PL::N, j, t);
  }
};

// ---------------------------------------------------------------------------
// the kernel: one CTA per packet of size N
// ---------------------------------------------------------------------------
// The whole time loop of one packet, run by the T = PL::T threads of one
// group (t = 0..T-1 inside the group, bar = the group's barrier id, smem =
// the group's spo1d_smem_bytes<R, PL, kTab>() bytes of shared memory).
template <typename R, class PL, bool kQuirk, int kTab>
__device__ __forceinline__ void spo_packet(const SpoArgs<R>& a, const SpoPacket pk, const int t,
                                           unsigned char* smem, const int bar) {
  constexpr int N = PL::N, P = PL::P, T = PL::T;
  constexpr int NW = (T + 31) / 32;
  using Th = SpoThread<R, PL>;
  using TB = Tab<R>;
  cpx<R>* bufs = reinterpret_cast<cpx<R>*>(smem);
  double2* cpart = reinterpret_cast<double2*>(bufs + Th::NBUF * N);  // [2][NW]
  TabStore<R, PL, kTab> tab;
  tab.init(cpart + 2 * NW);

  const int lane = t & 31, warp = t >> 5;
  const int base = pk.off;
  double2* cout = a.c_out + pk.c_off;

  Th th;
  th.bar = bar;
  th.init_twiddles(t);
  bool finite = true;  // C(t) samples written by this thread stayed finite

  cpx<R> v[P];
  double c0r = 0.0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const int x = base + Th::x_pos(t, j);
    const double2 p0 = a.psi_start ? a.psi_start[x] : a.psi0[x];
    c0r += p0.x * p0.x + p0.y * p0.y;
    v[j] = mk((R)p0.x, (R)p0.y);
    typename TB::phase_t kk{};
    if constexpr (!kQuirk) kk = a.tab.k[base + Th::final_pos(t, j)];
    tab.put(j, t, a.tab.g[x], kk, a.tab.w[x]);
  }
  // C(0) = <psi0|psi0> (a resumed run continues a series: its first sample
  // belongs to the previous segment)
  if (!a.psi_start) {
    double cr = c0r;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cr += __shfl_xor_sync(0xffffffffu, cr, o);
    if (lane == 0) cpart[warp] = make_double2(cr, 0.0);
    group_bar<T>(bar);
    if (t == 0) {
      double sr = 0.0;
      for (int i = 0; i < NW; ++i) sr += cpart[i].x;
      cout[0] = make_double2(sr, 0.0);
    }
    group_bar<T>(bar);
  }

  for (int step = 1; step <= a.nsteps; ++step) {
    // x-space phase
    if (step == 1) {
#pragma unroll
      for (int j = 0; j < P; ++j) v[j] = TB::apply(a.tab.h[base + Th::x_pos(t, j)], v[j]);
    } else {
#pragma unroll
      for (int j = 0; j < P; ++j) v[j] = TB::apply(tab.G(j, t), v[j]);
    }
    th.template forward<0>(v, bufs, t);
    // sum of the previous step's partial C(t): all partials are visible after
    // the first exchange barrier of this step
    if (T > 32 && t == 0 && step > 1) {
      const double2 c = sum_partials<NW>(cpart + ((step - 1) & 1) * NW);
      finite = finite && isfinite(c.x) && isfinite(c.y);
      cout[step - 1] = c;
    }
    // kinetic phase
    if constexpr (kQuirk) {
      // spofft.f:148-154 as written: V(I) uses the already updated U(I)
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const int f = base + Th::final_pos(t, j);
        const double c = a.kq_c[f], s = a.kq_s[f];
        const double un = c * (double)v[j].x + s * (double)v[j].y;
        const double vn = c * (double)v[j].y - s * un;
        v[j] = mk((R)(un * a.kq_scale), (R)(vn * a.kq_scale));
      }
    } else {
#pragma unroll
      for (int j = 0; j < P; ++j) v[j] = TB::apply(tab.K(j, t), v[j]);
    }
    th.template inverse<PL::S - 1>(v, bufs, t);
    // partial C(t) = sum w phi: the P products of a thread are summed in the
    // working precision (for FP32 a relative 1e-7 of a partial of size
    // ~1/N_threads), everything beyond the thread in FP64
    double cr, ci;
    {
      R pr = R(0), pi = R(0);
#pragma unroll
      for (int j = 0; j < P; ++j) {
        const typename TB::weight_t wj = tab.W(j, t);
        pr = fma(wj.x, v[j].x, fma(-wj.y, v[j].y, pr));
        pi = fma(wj.x, v[j].y, fma(wj.y, v[j].x, pi));
      }
      cr = (double)pr;
      ci = (double)pi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cr += __shfl_xor_sync(0xffffffffu, cr, o);
      ci += __shfl_xor_sync(0xffffffffu, ci, o);
    }
    if constexpr (T <= 32) {
      if (lane == 0) {
        finite = finite && isfinite(cr) && isfinite(ci);
        cout[step] = make_double2(cr, ci);
      }
    } else {
      if (lane == 0) cpart[(step & 1) * NW + warp] = make_double2(cr, ci);
    }
  }
  if constexpr (T > 32) {
    group_bar<T>(bar);
    if (t == 0 && a.nsteps > 0) {
      const double2 c = sum_partials<NW>(cpart + (a.nsteps & 1) * NW);
      finite = finite && isfinite(c.x) && isfinite(c.y);
      cout[a.nsteps] = c;
    }
  }
  // one count per packet whose C(t) went non-finite during the run
  if (!finite && a.nonfinite) atomicAdd(a.nonfinite, 1);
  // psi(TF) = hm . phi
  if (a.psi_out) {
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int x = base + Th::x_pos(t, j);
      cpx<R> o = (a.nsteps > 0) ? TB::apply(a.tab.hm[x], v[j]) : v[j];
      a.psi_out[x] = make_double2((double)o.x, (double)o.y);
    }
  }
}

// one CTA of PL::T threads per packet of one size class
template <typename R, class PL, bool kCap, bool kQuirk, int kTab, int kMinBlocks>
__global__ void __launch_bounds__(PL::T, kMinBlocks) spo1d_kernel(SpoArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  spo_packet<R, PL, kQuirk, kTab>(a, a.pk[blockIdx.x], threadIdx.x, smem_raw, 0);
}

template <typename R, class PL, int kTab>
constexpr size_t spo1d_smem_bytes() {
  return SpoThread<R, PL>::NBUF * sizeof(cpx<R>) * PL::N + 2 * sizeof(double2) * ((PL::T + 31) / 32) +
         TabStore<R, PL, kTab>::smem_bytes;
}

}  // namespace espec
