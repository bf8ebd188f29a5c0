// dropin.cu -- Fortran-callable drop-ins for eSPec's propagators PSPOFFT
// (pspofft.f:1-150; 1D/2D/3D), PSODFFT (psodfft.f:1-211; 1D/2D/3D), PLNZ
// (plnz.f:1-155; 1D/2D/3D), PSOD (psod.f:1-208; 1D/2D/3D), PPSOD
// (ppsod.f:1-470; PSOD with a laser pulse) and PPLNZ (pplnz.f:1-340; PLNZ
// with a laser pulse), 1D/2D/3D.
//
// Each call propagates one packet on the GPU through a one-packet plan and
// leaves in the caller's arrays what the reference routine leaves there:
// psi(TF) in U1/V1 (PSODFFT, PSOD: psi(TF) in U2/V2 and psi(TF-dt) in U1/V1), the
// kinetic table in TC, C(t) every LC steps in columns MPR/MPI of LNZVC, and
// INFO = 1 when the energy (or norm) drifted more than TOL percent.  With
// PRTCRL = '.YES' or '.PARTIAL' the partial auto-correlation table is written
// to standard output in the reference's formats; the energies and norms of
// its rows are computed on the GPU (EFFT4, eigenergfft.f:58-100).  The run is
// split at the printed steps and resumed from the state on the device.
//
// The arithmetic is the reference's, defects included: the in-place kinetic
// multiply of spofft.f:150-153 and the never-applied .SMOOTHW mask of
// sodfft.f:108, and PLNZ's cos-before-sin of sil.f:145-148.  Cases the GPU
// path does not cover (PSPOFFT: odd 1D sizes and sizes above 7252 points,
// 2D/3D axes other than 32..512 powers of two; PSODFFT: odd 1D sizes and
// sizes above 3626; PLNZ: order above 16) and
// device errors set INFO = 2 and write the reason to standard error; nothing
// is computed on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
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

// the table head of plnz.f:96-101: FORMAT 1011 of plnz.f:153
const char* kSilHead =
    " \n"
    " Partial auto-correlation function:\n"
    " ==================================\n"
    "\n"
    "          *t*       *Energy*        *Cr(t)*       *Ci(t)*    *|C(t)|^2*      *|C|*\n";

// the table head of psod.f:101-106 (its FORMAT 1011 titles the fifth column
// *|C(t)|^2*)
const char* kPsodHead =
    " \n"
    " Partial auto-correlation function:\n"
    " ==================================\n"
    "\n"
    "       *t/fs*       *E/a.u.*        *Cr(t)*       *Ci(t)*    *|C(t)|^2*      *|C|*\n";

enum Kind { kSpo, kSod, kSil, kPsod };

// One packet's propagation through a GPU plan: the segment, C(t) and energy
// calls of the plan type behind it.
struct Backend {
  std::function<int(int)> run;   // k steps from psi0, C(0) written
  std::function<int(int)> cont;  // k more steps from the current state
  std::function<int(int, double*, double*)> cvals;  // C samples 0..k of the last call
  std::function<int(double&, double&)> energy;     // E, sum |psi|^2 of the current state
};

struct DropIn {
  const char* name;
  Kind kind;
  // Fortran scalars
  bool absorb;
  int prt;  // 0 none, 1 '.PARTIAL', 2 '.YES'
  int lc, mpr, mpi, mxdct, n;
  double dt, ti, tf, tol;
  double* lnzvc;
  Backend be;
  double e0 = 0, f0 = 0;
  int* info;
  // text the reference prints inside step s (LNZ's order messages); "" if none
  std::function<std::string(int)> step_text;

  // INFO = 2: a case the GPU path does not run, or a device error
  int fail(const char* why) {
    std::fprintf(stderr, "espec_gpu %s: %s\n", name, why);
    *info = 2;
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
  // E and the printed norm: sqrt(FNR^2 + FNI^2) with FNI = 0 for the FFT
  // propagators (pspofft.f:96-98), FNR itself for PLNZ (plnz.f:91) and PSOD
  // (psod.f:95; squared in the rows of its loop, psod.f:183)
  int energies(double& e, double& fnt) {
    double nr;
    if (be.energy(e, nr)) return fail_lib();
    fnt = (kind == kSil || kind == kPsod) ? nr : std::sqrt(nr * nr);
    return 0;
  }
  // INFO drift test: PSPOFFT tests the norm only with an absorber
  // (pspofft.f:137-142), PSODFFT only without one (psodfft.f:178-183), PLNZ
  // always (plnz.f:137-138)
  // always (plnz.f:137-138); PSOD only without an absorber, with which its
  // INFO stays 0 (psod.f:184-189, 197-202)
  void drift(double et, double fnt) {
    if (kind == kPsod && absorb) return;
    const bool de = std::fabs((et - e0) / e0) * 1.0e2 > tol;
    const bool dn = std::fabs((fnt - f0) / f0) * 1.0e2 > tol;
    const bool norm_counts = kind == kSil || kind == kPsod || (kind == kSpo) == absorb;
    if (de || (norm_counts && dn)) *info = 1;
  }
  std::string row(double t, double e, double cr, double ci, double fnt) const {
    const double ct = (kind == kSil || kind == kPsod) ? cr * cr + ci * ci
                                                      : std::sqrt(cr * cr + ci * ci);
    return crl_row(t, e, cr, ci, ct, fnt);
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
    for (size_t si = 0; si < stops.size(); ++si) {
      const int stop = stops[si], k = stop - done;
      cre.resize(k + 1);
      cim.resize(k + 1);
      if (si == 0) {  // from psi0: writes C(0) as well
        if (be.run(k) || be.cvals(k, cre.data(), cim.data())) return fail_lib();
        store_c(0, cre[0], cim[0]);
        if (prt) {
          emit(kind == kSil ? kSilHead : (kind == kPsod ? kPsodHead : kCrlHead));
          emit(row(ti, e0, cre[0], cim[0], f0));
        }
      } else {
        if (be.cont(k) || be.cvals(k, cre.data(), cim.data())) return fail_lib();
      }
      for (int j = 1; j <= k; ++j) {
        store_c(done + j, cre[j], cim[j]);
        if (step_text) emit(step_text(done + j));
      }
      done = stop;
      if (k > 0 && printed(stop)) {
        double et, fnt;
        if (energies(et, fnt)) return -1;
        if (kind == kPsod && stop >= 2) fnt = fnt * fnt;  // psod.f:183
        if (checked(stop)) drift(et, fnt);
        emit(row(t_of(stop), et, cre[k], cim[k], fnt));
      }
    }
    return 0;
  }
};

// absorber of the GPU plan: the prefix tests of spofft.f:65,162 / sodfft.f:66,108
// (PSOD tests its own: sod.f:71, 78)
int absorber(bool absorb, const char* tp, size_t len) {
  if (!absorb) return ESPEC_ABS_NONE;
  if (fstr_is(tp, len, ".VOPTIC")) return ESPEC_ABS_VOPTIC;
  if (fstr_is(tp, len, ".SMOOTHW")) return ESPEC_ABS_SMOOTHW;
  return ESPEC_ABS_NONE;
}

// false (INFO = 2, reason on stderr) when DT is not positive or the run
// would take more than 1e9 steps: the step counts below assume both
bool common_scalars(DropIn& d, const int* absorb, const char* prtcrl, size_t prtcrl_len,
                    const int* lc, const int* mpi, const int* mpr, const int* mxdct, const int* n,
                    const double* dt, const double* ti, const double* tf, const double* tol,
                    double* lnzvc) {
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
  if (!(d.dt > 0.0) || !((d.tf - d.ti) / d.dt < 1.0e9)) {
    d.fail("DT must be positive and (TF - TI)/DT below 1e9");
    return false;
  }
  return true;
}

// the FFT propagators: one-packet espec_spo_plan
struct FftDropIn : DropIn {
  espec_spo_plan* plan = nullptr;
  espec_spond_plan* nd = nullptr;  // 2D/3D split operator
  ~FftDropIn() {
    espec_spo_destroy(plan);
    espec_spond_destroy(nd);
  }

  int setup_nd(int method, int ndim, const char* tpabsor, size_t tpabsor_len, const int* np,
               const double* sh, const double* sm, double* tc, const double* vpot,
               const double* vabc, const double* u, const double* v) {
    long npts = 1;
    for (int a = 0; a < ndim; ++a) npts *= np[a];
    if (npts != n) return fail("N differs from the product of NP");
    if (lc < 1) return fail("LC must be at least 1");
    // DIGT for 2D/3D as the reference computes it (dkeft.f:80-137)
    const int quirks = ESPEC_Q_DIGT_ND |
                       (method == ESPEC_SPO ? ESPEC_Q_SPO_INPLACE : ESPEC_Q_SOD_SMOOTHW);
    espec::digt_nd_table(ndim, np, sh, sm, quirks, tc);
    const int ab = absorber(absorb, tpabsor, tpabsor_len);
    if (espec_spond_create_method(&nd, method, ndim, np, sh, sm, dt, ESPEC_FP64, ab, quirks) ||
        espec_spond_load(nd, vpot, ab == ESPEC_ABS_NONE ? nullptr : vabc, u, v, ESPEC_MEM_HOST,
                         nullptr))
      return fail_lib();
    be.run = [this](int k) { return espec_spond_run(nd, k, nullptr); };
    be.cont = [this](int k) { return espec_spond_continue(nd, k, nullptr); };
    be.cvals = [this](int, double* cr, double* ci) {
      return espec_spond_results(nd, cr, ci, nullptr, nullptr, ESPEC_MEM_HOST, nullptr);
    };
    be.energy = [this](double& e, double& nr) {
      return espec_spond_energies(nd, &e, &nr, nullptr);
    };
    double fnt;
    if (energies(e0, fnt)) return -1;
    f0 = fnt;
    return 0;
  }

  int setup(int method, const char* dim, size_t dim_len, const char* tpabsor, size_t tpabsor_len,
            const int* np, const double* sh, const double* sm, double* tc, const double* vpot,
            const double* vabc, const double* u, const double* v) {
    const int ndim = fstr_is(dim, dim_len, ".2D") ? 2 : (fstr_is(dim, dim_len, ".3D") ? 3 : 1);
    if (ndim > 1) return setup_nd(method, ndim, tpabsor, tpabsor_len, np, sh, sm, tc, vpot, vabc, u, v);
    if (!fstr_is(dim, dim_len, ".1D")) return fail("DIM must be '.1D', '.2D' or '.3D'");
    if (np[0] != n) return fail("N differs from NP(1)");
    if (lc < 1) return fail("LC must be at least 1");
    // DIGT (dkeft.f:64-79): the kinetic table is an output of the reference
    espec::digt_1d(n, sh[0], sm[0], tc);
    const int ab = absorber(absorb, tpabsor, tpabsor_len);
    const int quirks = method == ESPEC_SPO ? ESPEC_Q_SPO_INPLACE : ESPEC_Q_SOD_SMOOTHW;
    if (espec_prop_create(&plan, 1, &n, sh, sm, dt, method, ESPEC_FP64, ab, quirks))
      return fail_lib();
    if (espec_spo_load(plan, vpot, ab == ESPEC_ABS_NONE ? nullptr : vabc, u, v, ESPEC_MEM_HOST,
                       nullptr))
      return fail_lib();
    be.run = [this](int k) { return espec_spo_run(plan, k, nullptr); };
    be.cont = [this](int k) { return espec_prop_continue(plan, k, nullptr); };
    be.cvals = [this](int, double* cr, double* ci) {
      return espec_spo_results(plan, cr, ci, nullptr, nullptr, ESPEC_MEM_HOST, nullptr);
    };
    be.energy = [this](double& e, double& nr) {
      return espec_prop_energies(plan, &e, &nr, nullptr);
    };
    // E0 and the norm of psi0 (the state of a freshly loaded plan)
    double fnt;
    if (energies(e0, fnt)) return -1;
    f0 = fnt;
    return 0;
  }
};

// gfortran list-directed text of LNZ's order messages (lnz.f:64-72)
std::string lnz_order_text(int nreort, int lmtreort, bool change) {
  char buf[256];
  std::string s = " Error NREORT > LMTREORT\n";
  std::snprintf(buf, sizeof buf, " NREORT=%12d   LMTREORT=%12d\n", nreort, lmtreort);
  s += buf;
  if (change) {
    s += " Modifing NREORT to correct value!\n";
    std::snprintf(buf, sizeof buf, " NREORT=%12d   LMTREORT=%12d\n", lmtreort, lmtreort);
    s += buf;
  }
  return s;
}

// ------------------------------------------------------------------------
// Shared by the pulse drop-ins (PPSOD, PPLNZ)
// ------------------------------------------------------------------------

// DIM of a grid drop-in: 1, 2 or 3; 0 if not one of those
int grid_dim(const char* dim, size_t len) {
  if (fstr_is(dim, len, ".1D")) return 1;
  if (fstr_is(dim, len, ".2D")) return 2;
  if (fstr_is(dim, len, ".3D")) return 3;
  return 0;
}

// EFC (ef.f:44-60) and its parameters in espec_pulse_field's order; -1 when
// the pulse is not known
int pulse_shape(const char* efc, size_t len, double e0, double tp, double omg, double t0,
                double td, double sni, int kl, double (&par)[6]) {
  int shape = -1;
  if (fstr_is(efc, len, ".GAUS")) shape = ESPEC_PULSE_GAUS;
  else if (fstr_is(efc, len, ".GGAUS")) shape = ESPEC_PULSE_GGAUS;
  else if (fstr_is(efc, len, ".SIN2")) shape = ESPEC_PULSE_SIN2;
  else if (fstr_is(efc, len, ".NONE") || fstr_is(efc, len, ".NULL")) shape = ESPEC_PULSE_NONE;
  const double p[6] = {e0, tp, omg, shape == ESPEC_PULSE_SIN2 ? td : t0, sni, (double)kl};
  for (int i = 0; i < 6; ++i) par[i] = p[i];
  return shape;
}

// the lines before a pulse table's column titles: a blank record, the title
// ('Auto-' when DIM .EQ. '.1D'), its rule and FORMAT 1011's leading empty record
std::string pulse_title(const char* dim, size_t len) {
  const bool one = len >= 3 && std::memcmp(dim, ".1D", 3) == 0 &&
                   std::string(dim + 3, len - 3).find_first_not_of(' ') == std::string::npos;
  return std::string(" \n") + (one ? " Auto-correlation function:\n"
                                    : " Partial auto-correlation function:\n") +
         " ==================================\n\n";
}

// the column titles common to both tables (FORMAT 1011 up to the groups)
const char* kPulseCols = "        *t/fs*     *ET/a.u.*      *E0/a.u.*      *Pr(t)*    *Pi(t)*   ";

// a grid plan and the device copy of the projection vectors, freed together
struct PulsePlan {
  espec_grid_plan* plan = nullptr;
  double* d_w = nullptr;
  int nw = 0;
  PulsePlan() = default;
  PulsePlan(const PulsePlan&) = delete;
  PulsePlan& operator=(const PulsePlan&) = delete;
  ~PulsePlan() {
    espec_grid_destroy(plan);
    if (d_w) cudaFree(d_w);
  }
  // W_k = LNZVC(1:N, KP+k), k = 1..nw (leading dimension MXDCT)
  bool load_w(const double* lnzvc, long mxdct, int kp, int count, long n) {
    nw = count;
    if (count <= 0) return true;
    if (cudaMalloc(&d_w, sizeof(double) * n * count) != cudaSuccess) return false;
    for (int k = 0; k < count; ++k)
      if (cudaMemcpy(d_w + (size_t)k * n, lnzvc + (size_t)(kp + k) * mxdct, sizeof(double) * n,
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    return true;
  }
};

// what a printed row needs from the state on the device: the energy with the
// field EF and without it, the norm, and <W_k|u>, <W_k|v> per vector
struct PulseRow {
  double et = 0, e0 = 0, fnr = 0;
  std::vector<double> pj;
  double pop(int k) const { return pj[2 * k] * pj[2 * k] + pj[2 * k + 1] * pj[2 * k + 1]; }
};

int measure_row(PulsePlan& pp, double ef, PulseRow& r) {
  double nr0;
  r.pj.assign(2 * (size_t)std::max(pp.nw, 1), 0.0);
  if (int rc = espec_grid_energies_at(pp.plan, ef, &r.et, &r.fnr, nullptr)) return rc;
  if (int rc = espec_grid_energies_at(pp.plan, 0.0, &r.e0, &nr0, nullptr)) return rc;
  if (pp.nw > 0) return espec_grid_project(pp.plan, pp.d_w, pp.nw, r.pj.data(), nullptr);
  return ESPEC_OK;
}

// FORMAT 1021 up to Ci: (1X,F14.6,3X,2(E12.6,3X),2(F8.5,3X) ...
std::string pulse_row_start(double t, const PulseRow& r, double cr, double ci) {
  return " " + fmt_f(t, 14, 6) + "   " + fmt_e(r.et, 12, 6) + "   " + fmt_e(r.e0, 12, 6) + "   " +
         fmt_f(cr, 8, 5) + "   " + fmt_f(ci, 8, 5);
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
  FftDropIn d;
  d.name = "PSPOFFT";
  d.kind = kSpo;
  d.info = info;
  if (!common_scalars(d, absorb, prtcrl, prtcrl_len, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol,
                      lnzvc))
    return;
  if (d.setup(ESPEC_SPO, dim, dim_len, tpabsor, tpabsor_len, np, sh, sm, tc, vpot, vabc, u1, v1))
    return;
  // DO T = TI+DT, TF+DT, DT (pspofft.f:110): T accumulates by DT
  const int nsteps = do_count(*ti + *dt, *tf + *dt, *dt);
  std::vector<double> tt(nsteps + 1, *ti);
  if (nsteps >= 1) tt[1] = *ti + *dt;
  for (int s = 2; s <= nsteps; ++s) tt[s] = tt[s - 1] + *dt;
  if (d.propagate(nsteps, [&](int s) { return tt[s]; }, [](int) { return true; })) return;
  const int rc = d.nd ? espec_spond_results(d.nd, nullptr, nullptr, u1, v1, ESPEC_MEM_HOST, nullptr)
                      : espec_spo_results(d.plan, nullptr, nullptr, u1, v1, ESPEC_MEM_HOST,
                                          nullptr);
  if (rc) {
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
  FftDropIn d;
  d.name = "PSODFFT";
  d.kind = kSod;
  d.info = info;
  if (!common_scalars(d, absorb, prtcrl, prtcrl_len, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol,
                      lnzvc))
    return;
  if (d.setup(ESPEC_SOD, dim, dim_len, tpabsor, tpabsor_len, np, sh, sm, tc, vpot, vabc, u1, v1))
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
  const bool bad =
      d.nd ? (espec_spond_results(d.nd, nullptr, nullptr, u2, v2, ESPEC_MEM_HOST, nullptr) ||
              espec_spond_previous(d.nd, u1, v1, ESPEC_MEM_HOST, nullptr))
           : (espec_spo_results(d.plan, nullptr, nullptr, u2, v2, ESPEC_MEM_HOST, nullptr) ||
              espec_prop_previous(d.plan, u1, v1, ESPEC_MEM_HOST, nullptr));
  if (bad) {
    d.fail_lib();
    return;
  }
  std::fflush(stdout);
}

// PLNZ: one espec_grid_plan (1D, 2D or 3D)
extern "C" void plnz_(const int* absorb, const int* change, const char* dim, const char* prtcrl,
                      const char* tpabsor, int* info, const int* lc, const int* lmtreort, int* mp,
                      const int* mpi, const int* mpr, const int* mxdct, const int* n,
                      const double* abstol, const double* dt, const double* ti, const double* tf,
                      const double* tol, const int* np, int* iwork, const double* shm,
                      const double* vpot, const double* vabc, double* u, double* v,
                      const double* xi, const double* xf, double* wu, double* wv, double* wp,
                      double* work, const double* var, double* lnzvc, size_t dim_len,
                      size_t prtcrl_len, size_t tpabsor_len) {
  (void)abstol; (void)iwork; (void)xi; (void)xf; (void)wu; (void)wv; (void)wp; (void)work;
  (void)var;
  DropIn d;
  d.name = "PLNZ";
  d.kind = kSil;
  d.info = info;
  if (!common_scalars(d, absorb, prtcrl, prtcrl_len, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol,
                      lnzvc))
    return;
  int ndim = 0;
  if (fstr_is(dim, dim_len, ".1D")) ndim = 1;
  if (fstr_is(dim, dim_len, ".2D")) ndim = 2;
  if (fstr_is(dim, dim_len, ".3D")) ndim = 3;
  if (!ndim) {
    d.fail("DIM must be '.1D', '.2D' or '.3D'");
    return;
  }
  long npts = 1;
  for (int a = 0; a < ndim; ++a) npts *= np[a];
  if (npts != *n) {
    d.fail("N differs from the product of NP");
    return;
  }
  if (d.lc < 1) {
    d.fail("LC must be at least 1");
    return;
  }
  // LNZ's order test (lnz.f:64-72): NREORT and M are both the caller's MP;
  // with *CHANGE the first call lowers it to LMTREORT for good
  const int mp_in = *mp;
  const bool clamp = mp_in > *lmtreort;
  const int m = clamp && *change ? *lmtreort : mp_in;
  if (m < 1 || m > 16) {
    d.fail("the GPU Lanczos order is limited to 1..16");
    return;
  }
  if (clamp) {
    const bool ch = *change != 0;
    const int lmt = *lmtreort;
    d.step_text = [mp_in, lmt, ch](int s) -> std::string {
      if (ch) return s == 1 ? lnz_order_text(mp_in, lmt, true) : std::string();
      const std::string one = lnz_order_text(mp_in, lmt, false);
      return one + one;  // both chains of the step
    };
  }
  // .SMOOTHW mask after each step (sil.f:171); any other absorber is ignored
  const int ab = d.absorb && fstr_is(tpabsor, tpabsor_len, ".SMOOTHW") ? ESPEC_ABS_SMOOTHW
                                                                        : ESPEC_ABS_NONE;
  espec_grid_plan* plan = nullptr;
  struct Guard {
    espec_grid_plan*& p;
    ~Guard() { espec_grid_destroy(p); }
  } guard{plan};
  if (espec_grid_create(&plan, ESPEC_SIL, ndim, np, shm, d.dt, m, ESPEC_FP64, ab,
                        ESPEC_Q_SIL_INPLACE) ||
      espec_grid_load(plan, vpot, vabc, u, v, ESPEC_MEM_HOST, nullptr)) {
    d.fail_lib();
    return;
  }
  d.be.run = [&](int k) { return espec_grid_run(plan, k, nullptr); };
  d.be.cont = [&](int k) { return espec_grid_continue(plan, k, nullptr); };
  d.be.cvals = [&](int, double* cr, double* ci) {
    return espec_grid_results(plan, cr, ci, nullptr, nullptr, ESPEC_MEM_HOST, nullptr);
  };
  d.be.energy = [&](double& e, double& nr) { return espec_grid_energies(plan, &e, &nr, nullptr); };
  double fnt;
  if (d.energies(d.e0, fnt)) return;
  d.f0 = fnt;
  // DO T = TI+DT, TF+DT, DT (plnz.f:104)
  const int nsteps = do_count(*ti + *dt, *tf + *dt, *dt);
  std::vector<double> tt(nsteps + 1, *ti);
  if (nsteps >= 1) tt[1] = *ti + *dt;
  for (int s = 2; s <= nsteps; ++s) tt[s] = tt[s - 1] + *dt;
  if (d.propagate(nsteps, [&](int s) { return tt[s]; }, [](int) { return true; })) return;
  // final energy and drift test (plnz.f:141-149)
  double et;
  if (d.energies(et, fnt)) return;
  d.drift(et, fnt);
  if (espec_grid_results(plan, nullptr, nullptr, u, v, ESPEC_MEM_HOST, nullptr) ||
      espec_grid_basis(plan, 1, lnzvc, *mxdct, ESPEC_MEM_HOST, nullptr)) {
    d.fail_lib();
    return;
  }
  if (clamp && *change) *mp = m;  // MP is modified through LNZ's NREORT argument
  std::fflush(stdout);
}

// PSOD: one espec_grid_plan (1D, 2D or 3D), method ESPEC_PSOD
extern "C" void psod_(const int* absorb, const char* dim, const char* prtcrl, const char* tpabsor,
                      int* info, const int* lc, const int* mp, const int* mpi, const int* mpr,
                      const int* mxdct, const int* n, const double* dt, const double* ti,
                      const double* tf, const double* tol, const int* np, const double* shm,
                      double* u1, double* u2, double* v1, double* v2, const double* xi,
                      const double* xf, const double* vpot, const double* vabc, double* work,
                      const double* var, double* lnzvc, size_t dim_len, size_t prtcrl_len,
                      size_t tpabsor_len) {
  (void)mp; (void)xi; (void)xf; (void)work; (void)var;
  DropIn d;
  d.name = "PSOD";
  d.kind = kPsod;
  d.info = info;
  if (!common_scalars(d, absorb, prtcrl, prtcrl_len, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol,
                      lnzvc))
    return;
  int ndim = 0;
  if (fstr_is(dim, dim_len, ".1D")) ndim = 1;
  if (fstr_is(dim, dim_len, ".2D")) ndim = 2;
  if (fstr_is(dim, dim_len, ".3D")) ndim = 3;
  if (!ndim) {
    d.fail("DIM must be '.1D', '.2D' or '.3D'");
    return;
  }
  long npts = 1;
  for (int a = 0; a < ndim; ++a) npts *= np[a];
  if (npts != *n) {
    d.fail("N differs from the product of NP");
    return;
  }
  if (d.lc < 1) {
    d.fail("LC must be at least 1");
    return;
  }
  int ab = ESPEC_ABS_NONE;  // sod.f:71-82
  if (d.absorb) {
    if (fstr_is(tpabsor, tpabsor_len, ".VOPTIC")) {
      ab = ESPEC_ABS_VOPTIC;
    } else if (fstr_is(tpabsor, tpabsor_len, ".SMOOTHW") || fstr_is(tpabsor, tpabsor_len, ".SMRS")) {
      ab = ESPEC_ABS_SMOOTHW;
    } else {
      d.fail("SOD propagation error: absorber type not '.VOPTIC', '.SMOOTHW' or '.SMRS'");
      return;
    }
  }
  espec_grid_plan* plan = nullptr;
  struct Guard {
    espec_grid_plan*& p;
    ~Guard() { espec_grid_destroy(p); }
  } guard{plan};
  if (espec_grid_create(&plan, ESPEC_PSOD, ndim, np, shm, d.dt, 0, ESPEC_FP64, ab,
                        ESPEC_Q_PSOD_COPY) ||
      espec_grid_load(plan, vpot, ab == ESPEC_ABS_NONE ? nullptr : vabc, u1, v1, ESPEC_MEM_HOST,
                      nullptr)) {
    d.fail_lib();
    return;
  }
  d.be.run = [&](int k) { return espec_grid_run(plan, k, nullptr); };
  d.be.cont = [&](int k) { return espec_grid_continue(plan, k, nullptr); };
  d.be.cvals = [&](int, double* cr, double* ci) {
    return espec_grid_results(plan, cr, ci, nullptr, nullptr, ESPEC_MEM_HOST, nullptr);
  };
  d.be.energy = [&](double& e, double& nr) { return espec_grid_energies(plan, &e, &nr, nullptr); };
  double fnt;
  if (d.energies(d.e0, fnt)) return;
  d.f0 = fnt;
  // start-up to T = TI+DT (psod.f:118-141), then DO T = TI+2*DT, TF+DT, DT
  // (psod.f:143); only rows of the loop run the drift test
  const int nsteps = 1 + do_count(*ti + 2 * *dt, *tf + *dt, *dt);
  std::vector<double> tt(nsteps + 1, *ti);
  tt[1] = *ti + *dt;
  if (nsteps >= 2) tt[2] = *ti + 2 * *dt;
  for (int s = 3; s <= nsteps; ++s) tt[s] = tt[s - 1] + *dt;
  if (d.propagate(nsteps, [&](int s) { return tt[s]; }, [](int s) { return s >= 2; })) return;
  // final energy and drift test after the loop (psod.f:192-202)
  double et;
  if (d.energies(et, fnt)) return;
  d.drift(et, fnt);
  if (espec_grid_results(plan, nullptr, nullptr, u2, v2, ESPEC_MEM_HOST, nullptr) ||
      espec_grid_previous(plan, u1, v1, ESPEC_MEM_HOST, nullptr)) {
    d.fail_lib();
    return;
  }
  std::fflush(stdout);
}

// PPSOD (ppsod.f:1-470): PSOD with the potential VP - DM EF(t) (chpot.f, ef.f)
// in every PSODAUX call, on a grid plan of method ESPEC_PSOD with the field
// table of espec_ppsod_field; without psod.f's restart-copy defect (PPSOD
// copies U0 into U1 after its start-up, ppsod.f:378-381).  Its table: FORMAT
// 1021 rows of T, ET (with the field), E0 (without), Cr, Ci, |C|^2, the
// populations |<W_k|psi>|^2 of W_k = LNZVC(., KP+k), and the norm; C(0) and
// the start-up sample are stored in LNZVC only inside the print test, as the
// reference does.
extern "C" void ppsod_(const int* absorb, const int* prtveff, const int* prteigvc2,
                       const int* prtpuls, const char* dim, const char* efc, const char* prtcrl,
                       const char* tpabsor, int* info, const int* lc, const int* mp,
                       const int* mpi, const int* mpr, const int* mxdct, const int* n,
                       const int* nshot, const int* npr_in, const int* kp, const int* nispg,
                       const double* e0, const double* t0, const double* td, const double* tp,
                       const double* omg, const double* sni, const int* kl, const double* dt,
                       const double* ti, const double* tf, const double* tol, const int* np,
                       const int* nd, const double* sh, const double* shm, double* u1,
                       double* u2, double* v1, double* v2, const double* xi, const double* xp,
                       const double* xf, const double* dm, double* vpot, const double* vabc,
                       double* work, const double* var, double* lnzvc, const int* prtregion,
                       const int* nreg, const double* range, const int* prtonlyreim,
                       size_t dim_len, size_t efc_len, size_t prtcrl_len, size_t tpabsor_len) {
  (void)mp; (void)nshot; (void)nd; (void)sh; (void)xi; (void)xp; (void)xf; (void)work;
  (void)var; (void)prtregion; (void)nreg; (void)range; (void)prtonlyreim; (void)prtveff;
  (void)prteigvc2; (void)prtpuls;
  *info = 0;
  auto fail = [&](const char* why) {
    std::fprintf(stderr, "espec_gpu PPSOD: %s\n", why);
    *info = 2;
  };
  const int ndim = grid_dim(dim, dim_len);
  if (!ndim) return fail("DIM must be '.1D', '.2D' or '.3D'");
  long npts = 1;
  for (int a = 0; a < ndim; ++a) npts *= np[a];
  if (npts != *n) return fail("N differs from the product of NP");
  if (*lc < 1) return fail("LC must be at least 1");
  if (!(*dt > 0.0) || !((*tf - *ti) / *dt < 1.0e9))
    return fail("DT must be positive and (TF - TI)/DT below 1e9");
  if (*npr_in > 6) return fail("NPR must be at most 6 (rdinput.f:660)");
  const int npr = std::max(*npr_in, 0);  // NPR < 1: no projections (ppsod.f:99-104)
  double par[6];
  const int shape = pulse_shape(efc, efc_len, *e0, *tp, *omg, *t0, *td, *sni, *kl, par);
  if (shape < 0) return fail("desired laser pulse wasn't found (ef.f:58-60)");
  int ab = ESPEC_ABS_NONE;  // sod.f:71-82
  if (*absorb) {
    if (fstr_is(tpabsor, tpabsor_len, ".VOPTIC")) ab = ESPEC_ABS_VOPTIC;
    else if (fstr_is(tpabsor, tpabsor_len, ".SMOOTHW") || fstr_is(tpabsor, tpabsor_len, ".SMRS"))
      ab = ESPEC_ABS_SMOOTHW;
    else return fail("SOD propagation error: absorber type not '.VOPTIC', '.SMOOTHW' or '.SMRS'");
  }
  const int prt = fstr_is(prtcrl, prtcrl_len, ".YES") ? 2
                  : (fstr_is(prtcrl, prtcrl_len, ".PARTIAL") ? 1 : 0);
  const long nn = *n;
  // the field of every PSODAUX call (ppsod.f:252-260, 378-386)
  std::vector<double> ef((size_t)std::max(8L, (long)((*tf - *ti) / *dt) + 8));
  const long ncalls = espec_ppsod_field(shape, par, *ti, *tf, *dt, ef.data(), (long)ef.size());
  if (ncalls < 2) return fail(espec_last_error());
  const int nsteps = (int)ncalls - 1;  // slot 1: the start-up; slot s >= 2: loop step s - 1
  std::vector<double> vp(vpot, vpot + nn);
  PulsePlan pp;
  if (espec_grid_create(&pp.plan, ESPEC_PSOD, ndim, np, shm, *dt, 0, ESPEC_FP64, ab, 0) ||
      espec_grid_load(pp.plan, vp.data(), ab == ESPEC_ABS_NONE ? nullptr : vabc, u1, v1,
                      ESPEC_MEM_HOST, nullptr) ||
      espec_grid_set_pulse(pp.plan, dm, ef.data(), ncalls, ESPEC_MEM_HOST))
    return fail(espec_last_error());
  // W_k = LNZVC(:, KP+k), k = 1..NPR (ppsod.f:99-104)
  if (!pp.load_w(lnzvc, *mxdct, *kp, npr, nn)) return fail("copy of the projection vectors");
  auto store = [&](long nc, double cr, double ci) {  // LNZVC(NC, MPR/MPI), NC from 1
    lnzvc[(nc - 1) + (long)(*mpr - 1) * *mxdct] = cr;
    lnzvc[(nc - 1) + (long)(*mpi - 1) * *mxdct] = ci;
  };
  double f0 = 0.0;
  // kind 0: the first row (sets F0), 1: the start-up row, 2: a loop row (drift
  // test, ppsod.f:440-444).  FORMAT 1021: ..., (3X,F8.6) for |C|^2, the
  // populations and the norm
  auto print_row = [&](double t, const PulseRow& m, double cr, double ci, int kind) {
    std::string row = pulse_row_start(t, m, cr, ci) + "   " + fmt_f(cr * cr + ci * ci, 8, 6);
    for (int k = 0; k < npr; ++k) row += "   " + fmt_f(m.pop(k), 8, 6);
    row += "   " + fmt_f(m.fnr, 8, 6) + "\n";
    if (kind == 2 && ab == ESPEC_ABS_NONE && std::fabs((m.fnr - f0) / f0) * 1.0e2 > *tol) *info = 1;
    if (kind == 0) f0 = m.fnr;
    emit(row);
  };
  // which slots print and which store C (ppsod.f:262-263, 388-396)
  std::vector<char> printed(nsteps + 1, 0), stored(nsteps + 1, 0);
  int mc = 1;
  if (prt == 2 || (prt == 1 && mc == *lc)) {
    printed[1] = 1;
    if (mc == *lc) {
      stored[1] = 1;
      mc = 0;
    }
  }
  for (int s = 2; s <= nsteps; ++s) {
    mc = mc + 1;
    if (mc == *lc) {
      mc = 0;
      stored[s] = 1;
    }
    if (prt == 2 || (prt == 1 && mc == 0)) printed[s] = 1;
  }
  long nc = 1;
  if (prt) {
    // the table head (ppsod.f:172-200): FORMAT 1011 or 1012 (two-digit indices)
    std::string head = pulse_title(dim, dim_len) + kPulseCols;
    const bool wide = *npr_in + *kp - 1 > 10;
    auto group = [&](const char* a, int i, const char* b, bool last) {
      char buf[32];
      std::snprintf(buf, sizeof buf, wide ? "%2d" : "%1d", i);
      std::string d(buf);
      if ((int)d.size() > (wide ? 2 : 1)) d = std::string(wide ? 2 : 1, '*');
      head += std::string(a) + d + b + (last ? "" : "   ");
    };
    group("*|P", *nispg - 1, "|^2*", false);
    for (int i = 1; i <= npr; ++i) group("*|P", i - 1 + *kp, "|^2*", false);
    group(" |c", *nispg - 1, "|^2 ", true);
    emit(head + "\n");
  }
  // the first row: psi0 with the potential before any CHPOT (ET = E0,
  // ppsod.f:158-201), printed once the run has given C(0)
  PulseRow first;
  if (prt && measure_row(pp, 0.0, first)) return fail(espec_last_error());
  // the run, split at the printed slots and resumed on the device
  std::vector<double> cre, cim;
  int done = 0;
  for (int s = 1; s <= nsteps; ++s) {
    if (!printed[s] && s != nsteps) continue;
    const int k = s - done;
    cre.resize(k + 1);
    cim.resize(k + 1);
    if ((done == 0 ? espec_grid_run(pp.plan, k, nullptr) : espec_grid_continue(pp.plan, k, nullptr)) ||
        espec_grid_results(pp.plan, cre.data(), cim.data(), nullptr, nullptr, ESPEC_MEM_HOST,
                           nullptr))
      return fail(espec_last_error());
    if (done == 0 && prt) {
      store(nc, cre[0], cim[0]);
      print_row(*ti, first, cre[0], cim[0], 0);
    }
    for (int j = 1; j <= k; ++j)
      if (stored[done + j]) store(++nc, cre[j], cim[j]);
    done = s;
    if (printed[s]) {
      // the time of slot s: TI + DT for the start-up, then T accumulating DT
      double t = *ti + *dt;
      for (int q = 2; q <= s; ++q) t = t + *dt;
      PulseRow m;
      if (measure_row(pp, ef[s], m)) return fail(espec_last_error());
      print_row(t, m, cre[k], cim[k], s >= 2 ? 2 : 1);
    }
  }
  if (done == 0) return fail("no steps");
  // psi(TF), psi(TF - dt), and VPOT as CHPOT leaves it
  if (espec_grid_results(pp.plan, nullptr, nullptr, u2, v2, ESPEC_MEM_HOST, nullptr) ||
      espec_grid_previous(pp.plan, u1, v1, ESPEC_MEM_HOST, nullptr))
    return fail(espec_last_error());
  for (long i = 0; i < nn; ++i) vpot[i] = vp[i] - dm[i] * ef[nsteps];
  std::fflush(stdout);
}

// PPLNZ (pplnz.f:1-340): PLNZ with the potential VP - DM EF(T) (chpot.f, ef.f)
// in each PLNZAUX step, DO T = TI+DT, TF+DT/2, DT, on a grid plan of method
// ESPEC_SIL with the field table of espec_pplnz_field and sil.f's in-place
// cos-before-sin.  Its table: FORMAT 1021 rows of T, ET (with the field), E0
// (without), Cr, Ci, CT(1..NPR) and the norm, where CT(1) = |C|^2 and CT(k+1)
// = |<W_k|psi>|^2 with W_k = LNZVC(., KP+k), k < NPR; on the first row the
// norm is printed squared (pplnz.f:146-147).  C(0) is stored in LNZVC only
// inside the print test, then every LC steps.
extern "C" void pplnz_(const int* absorb, const int* change, const int* prtveff,
                       const int* prteigvc2, const int* prtpuls, const char* dim, const char* efc,
                       const char* prtcrl, const char* tpabsor, int* info, const int* lc,
                       const int* lmtreort, int* mp, const int* mpi, const int* mpr,
                       const int* mxdct, const int* n, const int* nshot, const int* kl,
                       const int* npr_in, const int* kp, const double* abstol, const double* dt,
                       const double* ti, const double* tf, const double* tol, const double* e0,
                       const double* t0, const double* td, const double* tp, const double* omg,
                       const double* sni, const int* np, const int* nd, int* iwork,
                       const double* sh, const double* shm, double* vpot, const double* vabc,
                       double* u, double* v, const double* xi, const double* xf, const double* xp,
                       const double* dm, double* wu, double* wv, double* wp, double* work,
                       const double* var, double* lnzvc, size_t dim_len, size_t efc_len,
                       size_t prtcrl_len, size_t tpabsor_len) {
  (void)prtveff; (void)prteigvc2; (void)prtpuls; (void)nshot; (void)abstol; (void)nd;
  (void)iwork; (void)sh; (void)xi; (void)xf; (void)xp; (void)wu; (void)wv; (void)wp; (void)work;
  (void)var;
  *info = 0;
  auto fail = [&](const char* why) {
    std::fprintf(stderr, "espec_gpu PPLNZ: %s\n", why);
    *info = 2;
  };
  const int ndim = grid_dim(dim, dim_len);
  if (!ndim) return fail("DIM must be '.1D', '.2D' or '.3D'");
  long npts = 1;
  for (int a = 0; a < ndim; ++a) npts *= np[a];
  if (npts != *n) return fail("N differs from the product of NP");
  if (*lc < 1) return fail("LC must be at least 1");
  if (!(*dt > 0.0) || !((*tf - *ti) / *dt < 1.0e9))
    return fail("DT must be positive and (TF - TI)/DT below 1e9");
  if (*npr_in > 6) return fail("NPR must be at most 6 (rdinput.f:660)");
  const int npr = std::max(*npr_in, 0);
  const int nw = std::max(npr - 1, 0);  // printed projections: W_1 .. W_{NPR-1}
  double par[6];
  const int shape = pulse_shape(efc, efc_len, *e0, *tp, *omg, *t0, *td, *sni, *kl, par);
  if (shape < 0) return fail("desired laser pulse wasn't found (ef.f:58-60)");
  // LNZ's order test (lnz.f:64-72), as in PLNZ: with *CHANGE the first call
  // lowers MP to LMTREORT for good
  const int mp_in = *mp;
  const bool clamp = mp_in > *lmtreort;
  const int m = clamp && *change ? *lmtreort : mp_in;
  if (m < 1 || m > 16) return fail("the GPU Lanczos order is limited to 1..16");
  // .SMOOTHW mask after each step (sil.f:171); any other absorber is ignored
  const int ab = *absorb && fstr_is(tpabsor, tpabsor_len, ".SMOOTHW") ? ESPEC_ABS_SMOOTHW
                                                                     : ESPEC_ABS_NONE;
  const int prt = fstr_is(prtcrl, prtcrl_len, ".YES") ? 2
                  : (fstr_is(prtcrl, prtcrl_len, ".PARTIAL") ? 1 : 0);
  const long nn = *n;
  std::vector<double> ef((size_t)std::max(8L, (long)((*tf - *ti) / *dt) + 8));
  const long nfield = espec_pplnz_field(shape, par, *ti, *tf, *dt, ef.data(), (long)ef.size());
  if (nfield < 1) return fail(espec_last_error());
  const int nsteps = (int)nfield - 1;  // step s lands at T_s and uses EF(T_s)
  std::vector<double> vp(vpot, vpot + nn);
  PulsePlan pp;
  if (espec_grid_create(&pp.plan, ESPEC_SIL, ndim, np, shm, *dt, m, ESPEC_FP64, ab,
                        ESPEC_Q_SIL_INPLACE) ||
      espec_grid_load(pp.plan, vp.data(), ab == ESPEC_ABS_NONE ? nullptr : vabc, u, v,
                      ESPEC_MEM_HOST, nullptr) ||
      espec_grid_set_pulse(pp.plan, dm, ef.data(), nfield, ESPEC_MEM_HOST))
    return fail(espec_last_error());
  // W_k = LNZVC(:, KP+k) (pplnz.f:93-98), the printed ones
  if (!pp.load_w(lnzvc, *mxdct, *kp, nw, nn)) return fail("copy of the projection vectors");
  auto store = [&](long nc, double cr, double ci) {  // LNZVC(NC, MPR/MPI), NC from 1
    lnzvc[(nc - 1) + (long)(*mpr - 1) * *mxdct] = cr;
    lnzvc[(nc - 1) + (long)(*mpi - 1) * *mxdct] = ci;
  };
  double f0 = 0.0;
  // FORMAT 1021: ..., CT(1..NPR) = |C|^2 then the populations, FNT
  auto print_row = [&](double t, const PulseRow& r, double cr, double ci, bool first) {
    const double fnt = first ? r.fnr * r.fnr : r.fnr;
    std::string row = pulse_row_start(t, r, cr, ci);
    if (npr >= 1) row += "   " + fmt_f(cr * cr + ci * ci, 8, 6);
    for (int k = 0; k < nw; ++k) row += "   " + fmt_f(r.pop(k), 8, 6);
    row += "   " + fmt_f(fnt, 8, 6) + "\n";
    if (first) f0 = fnt;
    else if (!*absorb && std::fabs((fnt - f0) / f0) * 1.0e2 > *tol) *info = 1;
    emit(row);
  };
  // LNZ's messages of step s (both chains; with *CHANGE only the first call)
  auto step_text = [&](int s) -> std::string {
    if (!clamp) return std::string();
    if (*change) return s == 1 ? lnz_order_text(mp_in, *lmtreort, true) : std::string();
    const std::string one = lnz_order_text(mp_in, *lmtreort, false);
    return one + one;
  };
  // which steps store C and which print (pplnz.f:211-224)
  std::vector<char> printed(nsteps + 1, 0), stored(nsteps + 1, 0);
  int mc = 0;
  for (int s = 1; s <= nsteps; ++s) {
    mc = mc + 1;
    if (mc == *lc) {
      mc = 0;
      stored[s] = 1;
    }
    if (prt == 2 || (prt == 1 && mc == 0)) printed[s] = 1;
  }
  long nc = 1;
  PulseRow first;
  if (prt) {
    if (measure_row(pp, 0.0, first)) return fail(espec_last_error());
    // FORMAT 1011 (pplnz.f:331-332): groups (A3,I1,A4) joined by 3X
    std::string head = pulse_title(dim, dim_len) + kPulseCols;
    auto group = [&](const char* a, int i, bool last) {
      head += std::string(a) + (i >= 0 && i <= 9 ? std::string(1, (char)('0' + i)) : "*") +
              "|^2*" + (last ? "" : "   ");
    };
    for (int i = 1; i <= npr; ++i) group("*|P", i - 1, false);
    group("*|c", 0, true);
    emit(head + "\n");
  }
  std::vector<double> cre, cim;
  int done = 0;
  if (nsteps == 0 && prt) {  // no step: the first row alone
    std::vector<double> c0(2);
    if (espec_grid_run(pp.plan, 0, nullptr) ||
        espec_grid_results(pp.plan, &c0[0], &c0[1], nullptr, nullptr, ESPEC_MEM_HOST, nullptr))
      return fail(espec_last_error());
    store(nc, c0[0], c0[1]);
    print_row(*ti, first, c0[0], c0[1], true);
  }
  for (int s = 1; s <= nsteps; ++s) {
    if (!printed[s] && s != nsteps) continue;
    const int k = s - done;
    cre.resize(k + 1);
    cim.resize(k + 1);
    if ((done == 0 ? espec_grid_run(pp.plan, k, nullptr) : espec_grid_continue(pp.plan, k, nullptr)) ||
        espec_grid_results(pp.plan, cre.data(), cim.data(), nullptr, nullptr, ESPEC_MEM_HOST,
                           nullptr))
      return fail(espec_last_error());
    if (done == 0 && prt) {
      store(nc, cre[0], cim[0]);
      print_row(*ti, first, cre[0], cim[0], true);
    }
    std::string text;
    for (int j = 1; j <= k; ++j) {
      text += step_text(done + j);
      if (stored[done + j]) store(++nc, cre[j], cim[j]);
    }
    emit(text);
    done = s;
    if (printed[s]) {
      double t = *ti + *dt;  // the DO variable, accumulating DT
      for (int q = 2; q <= s; ++q) t = t + *dt;
      PulseRow r;
      if (measure_row(pp, ef[s], r)) return fail(espec_last_error());
      print_row(t, r, cre[k], cim[k], false);
    }
  }
  // psi(TF), the last step's Lanczos basis (LNZVC(., 1..MP), the V chain),
  // VPOT as CHPOT leaves it, MP as LNZ leaves it
  if (espec_grid_results(pp.plan, nullptr, nullptr, u, v, ESPEC_MEM_HOST, nullptr) ||
      (nsteps > 0 && espec_grid_basis(pp.plan, 1, lnzvc, *mxdct, ESPEC_MEM_HOST, nullptr)))
    return fail(espec_last_error());
  if (nsteps > 0)
    for (long i = 0; i < nn; ++i) vpot[i] = vp[i] - dm[i] * ef[nsteps];
  if (clamp && *change) *mp = m;
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
