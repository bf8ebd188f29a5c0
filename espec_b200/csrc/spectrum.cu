// spectrum.cu -- the spectrum stage of eSPec on the GPU, FP64, batched over
// packets: total correlation assembly (espec.f:1545-1576), lifetime
// broadening HWHM (hwhm.f:59-77), window and half swap of SPECTRUMTD
// (spectrumtd.f:58-81) fused into one pass, then the inverse DFT of FFTNT
// (cfft.f:6-106) as radix-2 Stockham passes (natural order in and out).
// Also the Fortran drop-ins hwhm_ and spectrumtd_ (with the printed table).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {
namespace {

constexpr double kHwhmScale = 1.5192676;           // hwhm.f:60-61
constexpr double kEnc = 1.519829846003e-1;         // spectrumtd.f:58
constexpr double kFate = 27.2113834;               // eV per hartree (spectrumtd.f)
constexpr double kTwoPi = 6.283185307179586476925287;

struct PrepArgs {
  int npk, mf;
  long ldc;               // stride of C(t) samples per packet (assemble) / of input (2^mf)
  const double2* in;      // C(t) samples (assemble) or the time signal
  int assemble;
  double dtf, tf;
  int hwhm;               // apply HWHM
  double dem, ta;         // -DE*1.5192676, TAL*1.5192676
  int window;             // 1: .SG
  double taux;            // TMAX^2 / ln(1/WP)^2
  double2* out;           // [npk][2^mf], halves swapped
};

// one element j of packet p: assembled (or read) C value, HWHM, window;
// written to the half-swapped position (spectrumtd.f:73-80)
__global__ void spec_prep_kernel(PrepArgs a) {
  const long N = 1L << a.mf;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= N * a.npk) return;
  const long p = gid / N, j = gid % N;
  double u, v;
  if (a.assemble) {
    // espec.f:1549-1563: C(-t) = C(t)* mirrored onto 2 MC points, MC = N/2
    const long mc = N / 2;
    const double2* c = a.in + p * a.ldc;
    if (j == 0) {
      u = c[mc - 1].x;
      v = -c[mc - 1].y;
    } else if (j <= mc) {
      u = c[mc - j].x;
      v = -c[mc - j].y;
    } else {
      u = c[j - mc].x;
      v = c[j - mc].y;
    }
  } else {
    const double2 z = a.in[p * a.ldc + j];
    u = z.x;
    v = z.y;
  }
  const double t = -a.tf + (double)j * a.dtf;
  if (a.hwhm) {  // hwhm.f:63-73
    double sn, cs;
    sincos(a.dem * t, &sn, &cs);
    const double cstl = exp(-fabs(t) * a.ta);
    const double ui = u;
    u = cs * u - sn * v;
    v = cs * v + sn * ui;
    u = cstl * u;
    v = cstl * v;
  }
  if (a.window) {  // spectrumtd.f:62-68
    const double cstl = exp(-(t * t) / a.taux);
    u = cstl * u;
    v = cstl * v;
  }
  const long js = (j + N / 2) % N;
  a.out[p * N + js] = make_double2(u, v);
}

// twiddles w_k = exp(+i twopi k / N), k < N/2 (the backward sign of FFTNT)
__global__ void spec_twiddle_kernel(double2* tw, long nh, double twopi_over_n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh) return;
  double s, c;
  sincos(twopi_over_n * (double)k, &s, &c);
  tw[k] = make_double2(c, s);
}

// one radix-2 Stockham pass (natural order after the last pass) of all
// packets; the last pass divides by N (cfft.f:102-105)
__global__ void spec_pass_kernel(const double2* x, double2* y, const double2* tw, int npk, int mf,
                                 int s, double scale) {
  const long N = 1L << mf, NH = N / 2;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= NH * npk) return;
  const long p = gid / NH, j = gid % NH;
  const long Ns = 1L << s;
  const long k = j & (Ns - 1);
  const double2* xp = x + p * N;
  double2* yp = y + p * N;
  const double2 a = xp[j], b0 = xp[j + NH];
  const double2 w = tw[k << (mf - 1 - s)];
  const double2 b = make_double2(b0.x * w.x - b0.y * w.y, b0.x * w.y + b0.y * w.x);
  const long d = ((j >> s) << (s + 1)) | k;
  yp[d] = make_double2((a.x + b.x) * scale, (a.y + b.y) * scale);
  yp[d + Ns] = make_double2((a.x - b.x) * scale, (a.y - b.y) * scale);
}

}  // namespace
}  // namespace espec

using namespace espec;

#define SPEC_CK(call)                                        \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return set_cuda_error(#call, e_); \
  } while (0)

// Device-side pipeline: in (device) -> spec (device, [npk][2^mf]); work is a
// device scratch of npk*2^mf double2 plus 2^(mf-1) twiddles.
extern "C" int espec_spectrum_dev(int npk, int mf, const void* in, long ld, int assemble,
                                  double dtf, double tf, double tal, double de, int window,
                                  double wp, int quirks, void* spec, void* work, void* stream) {
  if (npk <= 0 || mf < 0 || mf > 26 || !in || !spec || (mf > 0 && !work))
    return set_error(ESPEC_EINVAL, "bad spectrum arguments");
  if (window == 1 && !(wp > 0.0 && wp < 1.0))
    return set_error(ESPEC_EINVAL, "the .SG window needs 0 < WP < 1");
  cudaStream_t st = (cudaStream_t)stream;
  const long N = 1L << mf;
  PrepArgs a{};
  a.npk = npk;
  a.mf = mf;
  a.ldc = ld;
  a.in = (const double2*)in;
  a.assemble = assemble;
  a.dtf = dtf;
  a.tf = tf;
  a.hwhm = tal >= 0.0;
  a.dem = -de * kHwhmScale;
  a.ta = tal * kHwhmScale;
  a.window = window == 1;
  if (a.window) {
    const double tmax = N * dtf;
    const double l = std::log(1.0 / wp);
    a.taux = tmax * tmax / (l * l);
  }
  double2* bufs[2] = {(double2*)spec, (double2*)work};
  // the passes ping-pong; start in the buffer that makes the last pass land in spec
  int cur = (mf % 2 == 0) ? 0 : 1;
  a.out = bufs[cur];
  const long tot = N * npk;
  spec_prep_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(a);
  SPEC_CK(cudaGetLastError());
  if (mf == 0) return ESPEC_OK;  // FFTNT returns at N = 1 (cfft.f:39)
  // cfft.f:35 declares TWOPI with a default-real literal: single precision
  const double twopi = (quirks & ESPEC_Q_FFTNT_SP) ? (double)(float)kTwoPi : kTwoPi;
  double2* tw = (double2*)work + tot;
  spec_twiddle_kernel<<<(unsigned)((N / 2 + 255) / 256), 256, 0, st>>>(tw, N / 2, twopi / N);
  SPEC_CK(cudaGetLastError());
  const long nb = N / 2 * npk;
  for (int s = 0; s < mf; ++s) {
    const double scale = s == mf - 1 ? 1.0 / N : 1.0;
    spec_pass_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(bufs[cur], bufs[cur ^ 1], tw,
                                                                   npk, mf, s, scale);
    SPEC_CK(cudaGetLastError());
    cur ^= 1;
  }
  return ESPEC_OK;
}

extern "C" size_t espec_spectrum_work_bytes(int npk, int mf) {
  return sizeof(double2) * (((size_t)npk << mf) + ((size_t)1 << (mf > 0 ? mf - 1 : 0)));
}

// ---------------------------------------------------------------------------
// Fortran drop-ins
// ---------------------------------------------------------------------------
namespace {

// host arrays U, V of 2^M points through the device pipeline
int run_host(int mf, double dtf, double tf, double tal, double de, int window, double wp,
             int quirks, double* u, double* v) {
  const size_t N = (size_t)1 << mf;
  double2 *d_in = nullptr, *d_spec = nullptr, *d_work = nullptr;
  int rc = 0;
  auto cleanup = [&]() {
    if (d_in) cudaFree(d_in);
    if (d_spec) cudaFree(d_spec);
    if (d_work) cudaFree(d_work);
  };
  if ((rc = ck(cudaMalloc(&d_in, N * 16), "cudaMalloc")) ||
      (rc = ck(cudaMalloc(&d_spec, N * 16), "cudaMalloc")) ||
      (rc = ck(cudaMalloc(&d_work, espec_spectrum_work_bytes(1, mf)), "cudaMalloc"))) {
    cleanup();
    return rc;
  }
  if ((rc = ck(cudaMemcpy2D(d_in, 16, u, 8, 8, N, cudaMemcpyHostToDevice), "H2D")) ||
      (rc = ck(cudaMemcpy2D((char*)d_in + 8, 16, v, 8, 8, N, cudaMemcpyHostToDevice), "H2D")) ||
      (rc = espec_spectrum_dev(1, mf, d_in, (long)N, 0, dtf, tf, tal, de, window, wp, quirks,
                               d_spec, d_work, nullptr)) ||
      (rc = ck(cudaMemcpy2D(u, 8, d_spec, 16, 8, N, cudaMemcpyDeviceToHost), "D2H")) ||
      (rc = ck(cudaMemcpy2D(v, 8, (char*)d_spec + 8, 16, 8, N, cudaMemcpyDeviceToHost), "D2H"))) {
    cleanup();
    return rc;
  }
  cleanup();
  return ESPEC_OK;
}

std::string fmt_f12_7(double x) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.7f", x);
  std::string s(buf);
  if (s.size() > 12) {
    if (s.compare(0, 2, "0.") == 0) s.erase(0, 1);
    else if (s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
  }
  if (s.size() > 12) return std::string(12, '*');
  return std::string(12 - s.size(), ' ') + s;
}

}  // namespace

// HWHM (hwhm.f:1-80): TAL is scaled in place as the reference does
extern "C" void hwhm_(const int* m, const double* dt, const double* tf, double* tal,
                      const double* de, double* u, double* v) {
  if (*m < 0 || *m > 26) {
    std::fprintf(stderr, "espec_gpu HWHM: M out of range\n");
    return;
  }
  // only the lifetime/shift factors: no window, no transform
  const size_t N = (size_t)1 << *m;
  double2 *d_in = nullptr, *d_out = nullptr;
  if (cudaMalloc(&d_in, N * 16) != cudaSuccess || cudaMalloc(&d_out, N * 16) != cudaSuccess) {
    std::fprintf(stderr, "espec_gpu HWHM: device allocation failed\n");
    if (d_in) cudaFree(d_in);
    return;
  }
  PrepArgs a{};
  a.npk = 1;
  a.mf = *m;
  a.ldc = (long)N;
  a.in = d_in;
  a.dtf = *dt;
  a.tf = *tf;
  a.hwhm = 1;
  a.dem = -*de * kHwhmScale;
  a.ta = *tal * kHwhmScale;
  a.out = d_out;
  cudaMemcpy2D(d_in, 16, u, 8, 8, N, cudaMemcpyHostToDevice);
  cudaMemcpy2D((char*)d_in + 8, 16, v, 8, 8, N, cudaMemcpyHostToDevice);
  spec_prep_kernel<<<(unsigned)((N + 255) / 256), 256>>>(a);
  // prep writes half-swapped: read back with the halves exchanged
  const size_t h = N / 2;
  cudaError_t e = cudaGetLastError();
  if (N == 1) {
    cudaMemcpy2D(u, 8, d_out, 16, 8, 1, cudaMemcpyDeviceToHost);
    cudaMemcpy2D(v, 8, (char*)d_out + 8, 16, 8, 1, cudaMemcpyDeviceToHost);
  } else {
    cudaMemcpy2D(u, 8, d_out + h, 16, 8, h, cudaMemcpyDeviceToHost);
    cudaMemcpy2D(u + h, 8, d_out, 16, 8, h, cudaMemcpyDeviceToHost);
    cudaMemcpy2D(v, 8, (char*)(d_out + h) + 8, 16, 8, h, cudaMemcpyDeviceToHost);
    e = cudaMemcpy2D(v + h, 8, (char*)d_out + 8, 16, 8, h, cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) std::fprintf(stderr, "espec_gpu HWHM: %s\n", cudaGetErrorString(e));
  cudaFree(d_in);
  cudaFree(d_out);
  *tal = *tal * kHwhmScale;  // hwhm.f:61
}

// SPECTRUMTD (spectrumtd.f:1-116): window, swap, backward FFTNT on the GPU,
// then the printed spectrum table; DE < 0 is set to 0 in the caller's
// variable as the reference does
extern "C" void spectrumtd_(const char* tpwind, const int* m, const double* dt, const double* tf,
                            const double* wp, double* de, double* u, double* v,
                            size_t tpwind_len) {
  const int mf = *m;
  if (*de < 0.0) *de = 0.0;
  auto is = [&](const char* pat) {
    const size_t k = std::strlen(pat);
    return tpwind && tpwind_len >= k && std::memcmp(tpwind, pat, k) == 0;
  };
  int window = -1;
  if (is(".SG")) window = 1;
  else if (is(".NONE") || is(".NULL")) window = 0;
  if (window < 0) {  // spectrumtd.f:70-72 (the reference then stops)
    std::fputs("<<<>>> Windowing function error <<<>>>\n", stdout);
    std::fflush(stdout);
    return;
  }
  if (mf < 0 || mf > 26 ||
      run_host(mf, *dt, *tf, -1.0, 0.0, window, *wp, ESPEC_Q_FFTNT_SP, u, v) != ESPEC_OK) {
    std::fprintf(stderr, "espec_gpu SPECTRUMTD: %s\n", espec_last_error());
    return;
  }
  const std::string out = espec::spectrum_table(mf, *dt, *de, u, v);
  std::fwrite(out.data(), 1, out.size(), stdout);
  std::fflush(stdout);
}

namespace espec {
// spectrumtd.f:84-97 (list-directed head, FORMAT 1011 and 1021): the energy
// axis from -N/2 ENC, the FFTNT output from its second half on
std::string spectrum_table(int mf, double dt, double de, const double* u, const double* v) {
  const size_t N = (size_t)1 << mf;
  double enc = 1.0 / (N * dt) * kEnc;
  enc = enc * kFate;
  double en = -(double)N / 2.0 * enc;
  std::string out = " \n Spectrum:\n =========\n";
  out += "     *E (eV)*           *W*           *FFTr*          *FFTi*\n";
  auto row = [&](size_t i) {
    out += " " + fmt_f12_7(en + de) + "    " + fmt_f12_7(u[i]) + "    " + fmt_f12_7(u[i]) +
           "    " + fmt_f12_7(v[i]) + "\n";
    en = en + enc;
  };
  for (size_t i = N / 2; i < N; ++i) row(i);
  for (size_t i = 0; i < N / 2; ++i) row(i);
  return out;
}
}  // namespace espec
