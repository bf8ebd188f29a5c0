// dropin.cu -- Fortran-callable drop-ins for eSPec's FFT propagators
// PSPOFFT (pspofft.f:1-150) and PSODFFT (psodfft.f:1-211), 1D.
//
// Each call propagates one packet on the GPU through a one-packet plan and
// leaves in the caller's arrays what the reference routine leaves there:
// psi(TF) in U1/V1 (PSODFFT: psi(TF) in U2/V2 and psi(TF-dt) in U1/V1), the
// kinetic table in TC, C(t) every LC steps in columns MPR/MPI of LNZVC, and
// INFO = 1 when the energy (or norm) drifted more than TOL percent.  With
// PRTCRL = '.YES' or '.PARTIAL' the partial auto-correlation table is written
// to standard output in the reference's formats; the energies and norms of
// its rows are computed on the GPU (EFFT4, eigenergfft.f:58-100).  The run is
// split at the printed steps and resumed from the state on the device.
//
// The arithmetic is the reference's, defects included: the in-place kinetic
// multiply of spofft.f:150-153 and the never-applied .SMOOTHW mask of
// sodfft.f:108.  Cases the GPU path does not cover (DIM other than '.1D',
// packet sizes other than 256..4096 of the form 2^k or 3*2^k) set INFO = -1
// and write the reason to standard error; nothing is computed on the CPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace {

// CHARACTER*(*) argument s(1:k) .EQ. pat (pat has k characters)
bool fstr_is(const char* s, size_t len, const char* pat) {
  const size_t k = std::strlen(pat);
  return s && len >= k && std::memcmp(s, pat, k) == 0;
}

// real DO loop trip count of gfortran: max(0, INT((b - a + c) / c))
int do_count(double a, double b, double c) {
  const double x = (b - a + c) / c;
  return x > 0.0 ? (int)x : 0;
}

// ------------------------------------------------------------------------
// Fortran edit descriptors used by FORMAT 1021 (pspofft.f:148)
// ------------------------------------------------------------------------
std::string rjust(const std::string& s, int w) {
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

std::string nonfinite(double x, int w) {
  if (std::isnan(x)) return rjust("NaN", w);
  if (x > 0) return rjust(w >= 8 ? "Infinity" : "Inf", w);
  return rjust(w >= 9 ? "-Infinity" : "-Inf", w);
}

// Fw.d
std::string fmt_f(double x, int w, int d) {
  if (!std::isfinite(x)) return nonfinite(x, w);
  char buf[512];
  std::snprintf(buf, sizeof buf, "%.*f", d, x);
  std::string s(buf);
  if ((int)s.size() > w) {  // the optional leading zero goes first
    if (s.compare(0, 2, "0.") == 0) s.erase(0, 1);
    else if (s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
  }
  return rjust(s, w);
}

// Ew.d with a two-digit exponent field (three digits drop the 'E')
std::string fmt_e(double x, int w, int d) {
  if (!std::isfinite(x)) return nonfinite(x, w);
  std::string digits(d, '0');
  int e10 = 0;
  bool neg = std::signbit(x);
  if (x != 0.0) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(x));  // d.ddddde+XX
    std::string m(buf);
    const size_t epos = m.find('e');
    digits.clear();
    for (size_t i = 0; i < epos; ++i)
      if (m[i] != '.') digits.push_back(m[i]);
    e10 = std::atoi(m.c_str() + epos + 1) + 1;
  }
  char ex[16];
  if (std::abs(e10) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
  else std::snprintf(ex, sizeof ex, "%c%03d", e10 < 0 ? '-' : '+', std::abs(e10));
  std::string s = std::string(neg ? "-" : "") + "0." + digits + ex;
  if ((int)s.size() > w) s.erase(neg ? 1 : 0, 1);
  return rjust(s, w);
}

// FORMAT 1021: (1X,F14.8,3X,E12.6,2(4X,F10.7),4X,F10.8,4X,F8.6)
std::string crl_row(double t, double e, double cr, double ci, double ct, double fnt) {
  return " " + fmt_f(t, 14, 8) + "   " + fmt_e(e, 12, 6) + "    " + fmt_f(cr, 10, 7) + "    " +
         fmt_f(ci, 10, 7) + "    " + fmt_f(ct, 10, 8) + "    " + fmt_f(fnt, 8, 6) + "\n";
}

// the table head of pspofft.f:101-106 / psodfft.f:111-116 (a list-directed
// record starts with a blank, the empty one included; FORMAT 1011 opens with
// an empty record)
const char* kCrlHead =
    " \n"
    " Partial auto-correlation function:\n"
    " ==================================\n"
    "\n"
    "       *t/fs*       *E/a.u.*        *Cr(t)*       *Ci(t)*      *|C(t)|*      *|C|*\n";

void emit(const std::string& s) {
  std::fwrite(s.data(), 1, s.size(), stdout);
}

struct DropIn {
  const char* name;
  int method;
  // Fortran scalars
  bool absorb;
  int prt;  // 0 none, 1 '.PARTIAL', 2 '.YES'
  int lc, mpr, mpi, mxdct, n;
  double dt, ti, tf, tol;
  double* lnzvc;
  espec_spo_plan* plan = nullptr;
  double e0 = 0, f0 = 0;
  int* info;

  ~DropIn() { espec_spo_destroy(plan); }

  int fail(const char* why) {
    std::fprintf(stderr, "espec_gpu %s: %s\n", name, why);
    *info = -1;
    return -1;
  }
  int fail_lib() { return fail(espec_last_error()); }

  void store_c(int s, double cr, double ci) {  // LNZVC(NC, MPR/MPI), NC = 1 + s/LC
    if (s % lc != 0) return;
    const long nc = s / lc;  // zero-based row
    lnzvc[nc + (long)(mpr - 1) * mxdct] = cr;
    lnzvc[nc + (long)(mpi - 1) * mxdct] = ci;
  }
  bool printed(int s) const { return prt == 2 || (prt == 1 && s % lc == 0); }
  int energies(double& e, double& fnt) {
    double nr;
    if (espec_prop_energies(plan, &e, &nr, nullptr)) return fail_lib();
    fnt = std::sqrt(nr * nr);  // FNI = FCORREL(U,V) - FCORREL(V,U) = 0
    return 0;
  }
  // INFO drift test; the norm enters with an absorber in PSPOFFT
  // (pspofft.f:137-142) and without one in PSODFFT (psodfft.f:178-183)
  void drift(double et, double fnt) {
    const bool de = std::fabs((et - e0) / e0) * 1.0e2 > tol;
    const bool dn = std::fabs((fnt - f0) / f0) * 1.0e2 > tol;
    const bool norm_counts = (method == ESPEC_SPO) == absorb;
    if (de || (norm_counts && dn)) *info = 1;
  }

  // Steps 0..nsteps; t_of(s) gives the printed time of step s, checked(s)
  // whether a printed row also runs the drift test.
  template <class TOf, class Checked>
  int propagate(int nsteps, TOf t_of, Checked checked) {
    std::vector<int> stops;
    for (int s = 1; s <= nsteps; ++s)
      if (printed(s)) stops.push_back(s);
    if (stops.empty() || stops.back() != nsteps) stops.push_back(nsteps);
    std::vector<double> cre, cim;
    int done = 0;
    auto pull = [&](int k) -> int {  // C samples 0..k of the last segment
      cre.resize(k + 1);
      cim.resize(k + 1);
      if (espec_spo_results(plan, cre.data(), cim.data(), nullptr, nullptr, ESPEC_MEM_HOST, nullptr))
        return fail_lib();
      return 0;
    };
    for (size_t si = 0; si < stops.size(); ++si) {
      const int stop = stops[si], k = stop - done;
      if (si == 0) {  // from psi0: writes C(0) as well
        if (espec_spo_run(plan, k, nullptr)) return fail_lib();
        if (pull(k)) return -1;
        store_c(0, cre[0], cim[0]);
        if (prt) {
          emit(kCrlHead);
          emit(crl_row(ti, e0, cre[0], cim[0], std::sqrt(cre[0] * cre[0] + cim[0] * cim[0]), f0));
        }
      } else {
        if (espec_prop_continue(plan, k, nullptr)) return fail_lib();
        if (pull(k)) return -1;
      }
      for (int j = 1; j <= k; ++j) store_c(done + j, cre[j], cim[j]);
      done = stop;
      if (k > 0 && printed(stop)) {
        double et, fnt;
        if (energies(et, fnt)) return -1;
        const double cr = cre[k], ci = cim[k];
        if (checked(stop)) drift(et, fnt);
        emit(crl_row(t_of(stop), et, cr, ci, std::sqrt(cr * cr + ci * ci), fnt));
      }
    }
    return 0;
  }
};

// absorber of the GPU plan: the prefix tests of spofft.f:65,162 / sodfft.f:66,108
int absorber(bool absorb, const char* tp, size_t len, int method) {
  (void)method;  // PSODFFT's mask test never matches: the plan's ESPEC_Q_SOD_SMOOTHW
  if (!absorb) return ESPEC_ABS_NONE;
  if (fstr_is(tp, len, ".VOPTIC")) return ESPEC_ABS_VOPTIC;
  if (fstr_is(tp, len, ".SMOOTHW")) return ESPEC_ABS_SMOOTHW;
  return ESPEC_ABS_NONE;
}

int common_setup(DropIn& d, const int* absorb, const char* dim, size_t dim_len, const char* prtcrl,
                 size_t prtcrl_len, const char* tpabsor, size_t tpabsor_len, const int* lc,
                 const int* mpi, const int* mpr, const int* mxdct, const int* n, const double* dt,
                 const double* ti, const double* tf, const double* tol, const int* np,
                 const double* sh, const double* sm, double* tc, const double* vpot,
                 const double* vabc, const double* u, const double* v, double* lnzvc) {
  *d.info = 0;
  d.absorb = *absorb != 0;
  d.prt = fstr_is(prtcrl, prtcrl_len, ".YES") ? 2 : (fstr_is(prtcrl, prtcrl_len, ".PARTIAL") ? 1 : 0);
  d.lc = *lc;
  d.mpr = *mpr;
  d.mpi = *mpi;
  d.mxdct = *mxdct;
  d.n = *n;
  d.dt = *dt;
  d.ti = *ti;
  d.tf = *tf;
  d.tol = *tol;
  d.lnzvc = lnzvc;
  if (!fstr_is(dim, dim_len, ".1D")) return d.fail("only DIM = '.1D' runs on the GPU");
  if (np[0] != d.n) return d.fail("N differs from NP(1)");
  if (d.lc < 1) return d.fail("LC must be at least 1");
  // DIGT (dkeft.f:64-79): the kinetic table is an output of the reference
  espec::digt_1d(d.n, sh[0], sm[0], tc);
  const int kind = absorber(d.absorb, tpabsor, tpabsor_len, d.method);
  const int quirks = d.method == ESPEC_SPO ? ESPEC_Q_SPO_INPLACE : ESPEC_Q_SOD_SMOOTHW;
  if (espec_prop_create(&d.plan, 1, &d.n, sh, sm, d.dt, d.method, ESPEC_FP64, kind, quirks))
    return d.fail_lib();
  if (espec_spo_load(d.plan, vpot, kind == ESPEC_ABS_NONE ? nullptr : vabc, u, v, ESPEC_MEM_HOST,
                     nullptr))
    return d.fail_lib();
  // E0 and the norm of psi0 (the state of a freshly loaded plan)
  double fnt;
  if (d.energies(d.e0, fnt)) return -1;
  d.f0 = fnt;
  return 0;
}

}  // namespace

extern "C" void pspofft_(const int* absorb, const char* dim, const char* prtcrl,
                         const char* tpabsor, int* info, const int* lc, const int* mp,
                         const int* mpi, const int* mpr, const int* mxdct, const int* n,
                         const double* dt, const double* ti, const double* tf, const double* tol,
                         const int* np, const double* shm, const double* sh, const double* sm,
                         double* u1, double* v1, const double* xi, const double* xf, double* tc,
                         const double* vpot, const double* vabc, double* lnzvc, double* wrk1,
                         double* wrk2, const double* var, size_t dim_len, size_t prtcrl_len,
                         size_t tpabsor_len) {
  (void)mp; (void)shm; (void)xi; (void)xf; (void)wrk1; (void)wrk2; (void)var;
  DropIn d;
  d.name = "PSPOFFT";
  d.method = ESPEC_SPO;
  d.info = info;
  if (common_setup(d, absorb, dim, dim_len, prtcrl, prtcrl_len, tpabsor, tpabsor_len, lc, mpi, mpr,
                   mxdct, n, dt, ti, tf, tol, np, sh, sm, tc, vpot, vabc, u1, v1, lnzvc))
    return;
  // DO T = TI+DT, TF+DT, DT (pspofft.f:110): T accumulates by DT
  const int nsteps = do_count(*ti + *dt, *tf + *dt, *dt);
  std::vector<double> tt(nsteps + 1, *ti);
  if (nsteps >= 1) tt[1] = *ti + *dt;
  for (int s = 2; s <= nsteps; ++s) tt[s] = tt[s - 1] + *dt;
  if (d.propagate(nsteps, [&](int s) { return tt[s]; }, [](int) { return true; })) return;
  if (espec_spo_results(d.plan, nullptr, nullptr, u1, v1, ESPEC_MEM_HOST, nullptr)) {
    d.fail_lib();
    return;
  }
  std::fflush(stdout);
}

extern "C" void psodfft_(const int* absorb, const char* dim, const char* prtcrl,
                         const char* tpabsor, int* info, const int* lc, const int* mp,
                         const int* mpi, const int* mpr, const int* mxdct, const int* n,
                         const double* dt, const double* ti, const double* tf, const double* tol,
                         const int* np, const double* shm, const double* sh, const double* sm,
                         double* u1, double* u2, double* v1, double* v2, const double* xi,
                         const double* xf, double* tc, const double* vpot, const double* vabc,
                         double* wrkr, double* wrki, const double* var, double* lnzvc,
                         size_t dim_len, size_t prtcrl_len, size_t tpabsor_len) {
  (void)mp; (void)shm; (void)xi; (void)xf; (void)wrkr; (void)wrki; (void)var;
  DropIn d;
  d.name = "PSODFFT";
  d.method = ESPEC_SOD;
  d.info = info;
  if (common_setup(d, absorb, dim, dim_len, prtcrl, prtcrl_len, tpabsor, tpabsor_len, lc, mpi, mpr,
                   mxdct, n, dt, ti, tf, tol, np, sh, sm, tc, vpot, vabc, u1, v1, lnzvc))
    return;
  // start-up step at T = TI+DT (psodfft.f:120-147), then DO T = TI+2*DT,
  // TF+DT, DT (psodfft.f:154); only rows of the loop run the drift test
  const int nsteps = 1 + do_count(*ti + 2 * *dt, *tf + *dt, *dt);
  std::vector<double> tt(nsteps + 1, *ti);
  tt[1] = *ti + *dt;
  if (nsteps >= 2) tt[2] = *ti + 2 * *dt;
  for (int s = 3; s <= nsteps; ++s) tt[s] = tt[s - 1] + *dt;
  if (d.propagate(nsteps, [&](int s) { return tt[s]; }, [](int s) { return s >= 2; })) return;
  // final energy and drift test after the loop (psodfft.f:197-206)
  double et, fnt;
  if (d.energies(et, fnt)) return;
  d.drift(et, fnt);
  if (espec_spo_results(d.plan, nullptr, nullptr, u2, v2, ESPEC_MEM_HOST, nullptr) ||
      espec_prop_previous(d.plan, u1, v1, ESPEC_MEM_HOST, nullptr)) {
    d.fail_lib();
    return;
  }
  std::fflush(stdout);
}

extern "C" int espec_format_crl_row(double t, double e, double cr, double ci, double ct,
                                    double fnt, char* buf, int len) {
  if (!buf || len <= 0) return espec::set_error(ESPEC_EINVAL, "null buffer");
  const std::string s = crl_row(t, e, cr, ci, ct, fnt);
  if ((int)s.size() >= len) return espec::set_error(ESPEC_EINVAL, "buffer too short");
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return (int)s.size();
}
