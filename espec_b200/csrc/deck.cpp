// deck.cpp -- eSPec input decks run through the GPU: the driver (espec.f)
// from the input deck (rdinput.f) to the spectrum, for one packet with a
// tabulated potential and its eigenvector, or with an analytic .1D/.2D
// potential and computed eigenstates (time-dependent or time-independent
// formalism), or for a spectrum of a correlation function read back.
//
// Covered: **MAIN *DIMENSION (.1D/.2D/.3D), *POTENTIAL (.FILE; the analytic
// .1D/.2D forms of MAKECST with their initial and final constant records),
// *GRID_RANGES, *MASS, *TPCALC (.SPECTRUM .TD or .TI, .PROPAGATION,
// .CORRELATION, .ENERGY, .ONLYSPEC), *INIEIGVC (.GETR; .CALC on .1D and .2D
// grids), *CHANGE, *SHIFT_POTENTIAL, *PRTCRL, *MASS_FACTOR, *DONOTSTOP;
// **TI *TPDIAG (.MTRXDIAG, .LANCZS, .LANCZSG), *NIST, *NFST, *ABSTOL and an
// initial potential of its own; **TD *PROPAG (.PFSPO, .PFSOD, .PSIL, .PSOD,
// .PPSOD, .PPSIL/.PPLNZ), *PRPGSTATE, *TPTRANS .ONE, *PRPTOL, *ABSORBING,
// *PULSE_AND_DIPOLE (pulses .GAUS, .GGAUS, .SIN2, .NONE; dipoles .CONST,
// .EXP, .EXP+ (analytic decks), .READ (a file as RDPTE reads it), .NONE,
// .NULL), *NPROJECTIONS (on the computed states; with .GETR on LNZVC(., 1)
// only, KP = 0), *NSHOT; **SPECTRUM *FOURIER, *WINDOWING, *HWHM.  Print and
// output-file switches (*PRTPOT, *PRTEIGVC, ...) are accepted and ignored:
// no files are written (nor initial_spc.aux or the unit-21 table of .EXP+).
// *TPCALC .COLLISION starts a .1D run from a Gaussian wave packet with a
// momentum (**TI *COLLISION_ENERGY, *SIZE_OF_GAUSSIAN, *INIT_POSSITION).
// Anything else -- 3D computed states, several transitions, 2D collisions,
// .2DC operators -- is refused with a message: there is no CPU path.
//
// The run follows espec.f: the .FILE reads of RDPTE / RDPT (rdpte.f, rdpt.f:
// eigenvector block, then potential block, optionally shifted to its
// minimum) or, for .CALC, the potentials of GVPOT and the eigenstates of the
// initial one (initial_state below),
// SH = (XF - XI)/(NP - 1) and SHM = 1/(24 m SH^2) per axis, the C(t)
// stride NC and the final time of espec.f:1328-1353, the absorber table of
// ABSORBINGBC (absorb.f:62-205), the propagator drop-in (which prints the
// partial auto-correlation table), the total correlation of espec.f:1545-1576
// printed as FORMAT 1041/1042, and HWHM / SPECTRUMTD (espec.f:1596-1606).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "espec_gpu.h"
#include "espec_internal.h"

#include <cuda_runtime.h>

namespace {

const double kAmu = 1.836152667539e3;  // espec.f:614
const double kA0A = 5.291772083e-1;    // angstrom per bohr (espec.f:67)

struct DeckError {
  std::string what;
};

std::string upper(std::string s) {
  for (char& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// free-format numbers of one record, up to a '/' (Fortran list-directed
// input; D exponents accepted)
std::vector<double> numbers(const std::string& line) {
  std::string s = line.substr(0, line.find('/'));
  for (char& c : s)
    if (c == 'D' || c == 'd') c = 'E';
    else if (c == ',') c = ' ';
  std::istringstream in(s);
  std::vector<double> v;
  std::string tok;
  while (in >> tok) {
    char* end = nullptr;
    const double x = std::strtod(tok.c_str(), &end);
    if (end == tok.c_str()) break;
    v.push_back(x);
  }
  return v;
}

bool starts(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

// One keyword's records, as the lines that follow it (comments after '!'
// removed, blank lines skipped).
struct Deck {
  std::map<std::string, std::map<std::string, std::vector<std::string>>> sec;
  // the keyword lines themselves (rdinput.f tests columns past the keyword,
  // e.g. '*GRID_RANGES au')
  std::map<std::string, std::map<std::string, std::string>> head;
  const std::vector<std::string>* get(const char* s, const char* k) const {
    auto a = sec.find(s);
    if (a == sec.end()) return nullptr;
    auto b = a->second.find(k);
    return b == a->second.end() ? nullptr : &b->second;
  }
};

// rdinput.f tests keyword lines by prefix, in this order per section (so
// '*MASSES' is *MASS, '*MASS_FACTORS' *MASS_FACTOR, '*GRID_RANGES_au'
// *GRID_RANGES); a line no prefix matches keeps its own name
std::string canon_key(const std::string& section, const std::string& key) {
  static const std::map<std::string, std::vector<std::string>> kOrder = {
      {"**MAIN",
       {"*TITLE", "*TPCALC", "*DIMENSION", "*GRID_CUT", "*TPTRANS", "*NREORT",
        "*INITIAL_POTENTIAL", "*FINAL_POTENTIAL", "*POTENTIAL", "*GRID_RANGES", "*INIEIGVC",
        "*MASS_FACTOR", "*MASS", "*SCALING_FA", "*CROSS_TERM", "*SEED", "*NSHOT", "*CHANGE",
        "*SHIFT_POTENTIAL", "*PRTEIGVC2", "*PRTREGION", "*PRTONLYREIM", "*PRTEIGVC", "*PRTPOT",
        "*PRTVEFF", "*PRTPULSE", "*PRTDIPOLE", "*DONOTSTOP", "*PRTCRL"}},
      {"**TI",
       {"*INITIAL_POTENTIAL", "*INITIAL_CONDITION", "*INITIAL_WP", "*INITIAL_WF",
        "*INITIAL_WAVE_FUNCTION", "*WAVE_FUNCTION", "*WAVE_PACKET", "*POTENTIAL", "*TPDIAG",
        "*NIST", "*ABSTOL", "*SEED", "*MAXINT", "*COLLISION_ENERGY", "*GRID_RANGES",
        "*INIT_POSSITION", "*SIZE_OF_GAUSSIAN"}},
      {"**TD",
       {"*PROPAG", "*FINAL_POTENTIAL", "*GRID_RANGES", "*ABSORBING", "*PULSE_AND_DIPOLE",
        "*PRPGSTATE", "*TPTRANS", "*PRPTOL", "*NSHOT", "*NPROJECTIONS", "*FOURIER"}},
      {"**SPECTRUM", {"*FOURIER", "*WINDOWING", "*HWHM"}}};
  auto it = kOrder.find(section);
  if (it == kOrder.end()) return key;
  for (const std::string& p : it->second)
    if (starts(key, p.c_str())) return p;
  return key;
}

Deck parse_deck(const std::string& text) {
  Deck d;
  std::istringstream in(text);
  std::string line, section, key;
  while (std::getline(in, line)) {
    const size_t bang = line.find('!');
    if (bang != std::string::npos) line = line.substr(0, bang);
    const std::string t = trim(line);
    if (t.empty()) continue;
    if (starts(t, "**") && t.size() > 2 && std::isalpha((unsigned char)t[2])) {
      section = upper(t.substr(0, t.find_first_of(" \t")));
      d.sec[section];
      key.clear();
    } else if (t[0] == '*') {
      if (section.empty() || starts(t, "**")) continue;  // title lines
      key = canon_key(section, upper(t.substr(0, t.find_first_of(" \t"))));
      d.sec[section][key];
      d.head[section][key] = t;
    } else if (!section.empty() && !key.empty()) {
      d.sec[section][key].push_back(t);
    }
  }
  return d;
}

// .FILE potential: title, NT eigenvector records, title, NT potential records
// (rdpte.f:39-58, rdpt.f:40-62), coordinates listed last axis first
struct FileData {
  std::vector<double> psi, vpot;
  std::vector<double> psi_im;  // a complex initial state (.COLLISION); empty: real
  double xi[3] = {0, 0, 0}, xf[3] = {0, 0, 0};
};

// one block of RDPTE / RDPT: a title record, then nt records of nd
// coordinates (last axis first) and a value; XI, XF from the first and last
void read_block(std::ifstream& f, const std::string& path, int nt, int nd, std::vector<double>& out,
                double* xi, double* xf) {
  std::string line;
  out.resize(nt);
  if (!std::getline(f, line)) throw DeckError{"reading file error: " + path};
  for (int j = 0; j < nt; ++j) {
    if (!std::getline(f, line)) throw DeckError{"reading file error: " + path};
    const std::vector<double> v = numbers(line);
    if ((int)v.size() < nd + 1) throw DeckError{"reading file error: " + path};
    out[j] = v[nd];
    if (j == 0)
      for (int a = 0; a < nd; ++a) xi[a] = v[nd - 1 - a];
    if (j == nt - 1)
      for (int a = 0; a < nd; ++a) xf[a] = v[nd - 1 - a];
  }
}

FileData read_file(const std::string& path, int nt, int nd, bool shiftp) {
  std::ifstream f(path);
  if (!f) throw DeckError{"potential input file \"" + path + "\" cannot be opened"};
  FileData r;
  read_block(f, path, nt, nd, r.psi, r.xi, r.xf);
  read_block(f, path, nt, nd, r.vpot, r.xi, r.xf);  // RDPT sets XI, XF again
  if (shiftp) {
    double vmin = r.vpot[0];
    for (double x : r.vpot) vmin = x < vmin ? x : vmin;
    for (double& x : r.vpot) x = x - vmin;
  }
  return r;
}

// ABSORBINGBC (absorb.f:62-205) on the grid
std::vector<double> absorber_table(int nd, const int* np, const std::string& tp, const double* al,
                                   const double* ar, const double* sh, const double* xi,
                                   const double* xf, const double* voi) {
  long n = 1;
  for (int a = 0; a < nd; ++a) n *= np[a];
  std::vector<double> v(n, 0.0);
  if (nd == 1) {
    for (long i = 0; i < n; ++i) {
      const double x = xi[0] + (double)i * sh[0];
      double r;
      if (starts(tp, ".SMOOTHW")) {
        if (x < al[0])
          r = std::exp(voi[0] * std::pow(x - al[0], voi[1]) / (x + sh[0] - xi[0]));
        else if (x > ar[0])
          r = std::exp(-voi[0] * (x - ar[0]) / std::pow(xf[0] + sh[0] - x, voi[1]));
        else
          r = 1.0;
      } else if (starts(tp, ".SMRS")) {
        r = x < al[0] ? 1.0 - voi[0] * (x - al[0]) * (x - al[0])
                      : (x > ar[0] ? 1.0 - voi[0] * (x - ar[0]) * (x - ar[0]) : 1.0);
      } else if (starts(tp, ".VOPTIC_LINEAR")) {
        r = x < al[0] ? -voi[0] * (x - al[0]) / (x + sh[0] - xi[0])
                      : (x > ar[0] ? voi[0] * (x - ar[0]) / (xf[0] + sh[0] - x) : 0.0);
      } else if (starts(tp, ".VOPTIC_KOSLOFF")) {
        r = x < al[0] ? voi[0] / std::cosh(xi[0] - al[0] / voi[1])
                      : (x > ar[0] ? voi[0] / std::cosh(xf[0] - al[0] / voi[1]) : 0.0);
      } else if (starts(tp, ".VOPTIC_POLIN")) {
        r = x < al[0] ? voi[0] * std::pow(x - al[0], voi[1])
                      : (x > ar[0] ? voi[0] * std::pow(x - ar[0], voi[1]) : 0.0);
      } else {
        throw DeckError{"absorber " + tp + " is not defined for .1D (absorb.f)"};
      }
      v[i] = r;
    }
    return v;
  }
  if (nd == 2 && starts(tp, ".SMOOTHW")) {
    for (int j = 0; j < np[1]; ++j) {
      const double y = xi[1] + (double)j * sh[1];
      for (int i = 0; i < np[0]; ++i) {
        const double x = xi[0] + (double)i * sh[0];
        double r;
        if (x < al[0])
          r = std::exp(voi[0] * (x - al[0]) / (x + sh[0] - xi[0]));
        else if (y < al[1])
          r = std::exp(voi[1] * (y - al[1]) / (y + sh[1] - xi[1]));
        else if (x > ar[0])
          r = std::exp(-voi[0] * (x - ar[0]) / (xf[0] + sh[0] - x));
        else if (y > ar[1])
          r = std::exp(-voi[1] * (y - ar[1]) / (xf[1] + sh[1] - y));
        else
          r = 1.0;
        v[i + (long)np[0] * j] = r;
      }
    }
    return v;
  }
  throw DeckError{"the reference has no absorber " + tp + " for this dimension (absorb.f:196-210)"};
}

// gfortran's real DO loop trip count: max(0, INT((b - a + c) / c))
int do_count_real(double a, double b, double c) {
  const double x = (b - a + c) / c;
  return x > 0.0 ? (int)x : 0;
}

// FORMAT 1003: (/,3X,A68) -- A68 right-justifies a shorter string
void msg1003(const char* s) {
  std::string t(s);
  if (t.size() < 68) t = std::string(68 - t.size(), ' ') + t;
  std::printf("\n   %s\n", t.substr(0, 68).c_str());
}

// list-directed REAL*8 as the reference's executable writes it: one blank,
// then 1PG23.15E3 (F form with 15 significant digits and 5 trailing blanks
// for 0.1 <= |x| < 1e15, else 1.ddd...E+xxx)
std::string list_real(double x) {
  char buf[64];
  const double ax = std::fabs(x);
  if (ax != 0.0 && (ax < 0.1 || ax >= 1e15)) {
    std::snprintf(buf, sizeof buf, "%.15E", x);
    std::string s(buf);
    const size_t e = s.find('E');
    const int ex = std::atoi(s.c_str() + e + 1);
    char eb[16];
    std::snprintf(eb, sizeof eb, "E%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    s = s.substr(0, e) + eb;
    return " " + std::string(s.size() < 23 ? 23 - s.size() : 0, ' ') + s;
  }
  const int k = ax == 0.0 ? 0 : (int)std::floor(std::log10(ax)) + 1;
  std::snprintf(buf, sizeof buf, "%.*f", 15 - (k > 0 ? k : 0), x);
  std::string s(buf);
  return " " + std::string(s.size() < 18 ? 18 - s.size() : 0, ' ') + s + "     ";
}

// Fortran Ew.d: 0.ddd...E+xx right-justified in w (the leading 0 dropped
// when the sign leaves no room for it)
std::string fort_e(double x, int w, int d) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.*E", d - 1, x);  // one digit before the point
  std::string s(buf);
  const bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  const size_t e = s.find('E');
  const int ex = x == 0.0 ? 0 : std::atoi(s.c_str() + e + 1) + 1;
  std::string digits = s.substr(0, 1) + s.substr(2, e - 2);
  char eb[16];
  std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
  std::string out = "0." + digits + eb;
  if (neg) out = "-" + out;
  if ((int)out.size() > w && neg) out = "-" + out.substr(2);
  if ((int)out.size() > w) return std::string(w, '*');
  return std::string(w - out.size(), ' ') + out;
}

// MAKECST (makecst.f:82-340) for a .1D or .2D deck: the constants of an
// analytic potential to atomic units, the first prefix that matches deciding,
// with its FORMAT 1020/1031/1041/1051/1061/1071 lines.  sm: the masses in
// electron masses.
void makecst(int nd, const std::string& potch, const double* sm, std::vector<double>& c) {
  const double ffreq = 4.556335252750e-6, ccgs = 2.99792458e10, eev = 27.211383411;
  const double tau = 2.4188843243e-17, twopi = 6.2831853071795864769252867663;
  const double ecm = 2.19474631371017e5, pi = 3.14159265358979323846;
  const double sm1 = sm[0];
  c.resize(14, 0.0);
  auto is = [&](const char* p) { return starts(potch, p); };
  auto l1031 = [&](int i, double a, double b) {
    std::printf(" Re_%d/a.u. = %s; K_%d/a.u. = %s;\n", i, fort_e(a, 12, 6).c_str(), i,
                fort_e(b, 12, 6).c_str());
  };
  auto l1041 = [&](int i, double a, double b, double d) {
    std::printf(" Re_%d/a.u. = %s; alpha_%d/a.u. = %s; D_%d/a.u. = %s\n", i,
                fort_e(a, 12, 6).c_str(), i, fort_e(b, 12, 6).c_str(), i,
                fort_e(d, 12, 6).c_str());
  };
  auto l1051i = [&](int i, double a, double b, double d) {
    std::printf(" R(min)_%d/a.u. = %s; R(max)_%d/a.u. = %s; Const_%d/a.u. = %s\n", i,
                fort_e(a, 12, 6).c_str(), i, fort_e(b, 12, 6).c_str(), i,
                fort_e(d, 12, 6).c_str());
  };
  auto l1051 = [&]() { l1051i(1, c[0], c[1], c[2]); };
  auto l1061 = [&]() { std::printf(" Const_1/a.u. = %s\n", fort_e(c[0], 12, 6).c_str()); };
  const char* au = " These parameters were already inputed in a.u.\n";
  const char* bad = "<<<>>> Potential parameter converting error <<<>>>\n";
  auto sq = [](double x) { return x * x; };
  if (nd == 2) {
    if (is(".OHS")) {
      const double fk1 = sq(((c[1] * ccgs) * tau) * twopi) * sm[0];
      const double fk2 = sq(((c[3] * ccgs) * tau) * twopi) * sm[1];
      c[0] = c[0] / kA0A;
      c[2] = c[2] / kA0A;
      c[1] = fk1;
      c[3] = fk2;
      l1031(1, c[0], c[1]);
      l1031(2, c[2], c[3]);
    } else if (is(".LSM_au")) {
      std::printf("%s", au);
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[0], c[3], c[4]);
      l1041(3, c[5], c[6], c[7]);
    } else if (is(".LSM")) {
      c[0] = c[0] / kA0A;
      c[5] = c[5] / kA0A;
      c[1] = c[1] * kA0A;
      c[3] = c[3] * kA0A;
      c[6] = c[6] * kA0A;
      c[2] = c[2] / ecm;
      c[4] = c[4] / ecm;
      c[7] = c[7] / ecm;
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[0], c[3], c[4]);
      l1041(3, c[5], c[6], c[7]);
    } else if (is(".LS_au")) {
      std::printf("%s", au);
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[0], c[3], c[4]);
    } else if (is(".LS")) {
      c[0] = c[0] / kA0A;
      c[1] = c[1] * kA0A;
      c[3] = c[3] * kA0A;
      c[2] = c[2] / ecm;
      c[4] = c[4] / ecm;
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[0], c[3], c[4]);
    } else if (is(".LBH")) {  // .LBH and .LBH_CC
      std::printf(" Not implemented!\n");
      throw DeckError{"potential " + potch + ": MAKECST stops (not implemented, makecst.f)"};
    } else if (is(".LEPS_CC_Dalpha_au") || is(".LEPS_Dalpha_au")) {
      std::printf("%s", au);
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[3], c[4], c[5]);
      l1041(3, c[6], c[7], c[8]);
      std::printf(" a = %s; b = %s; c = %s\n", fort_e(c[9], 10, 4).c_str(),
                  fort_e(c[10], 10, 4).c_str(), fort_e(c[11], 10, 4).c_str());
      c[12] = pi * c[12] / 1.8e2;
      std::printf(" Angle (rad) =%s\n", list_real(c[12]).c_str());
    } else if (is(".LEPS_CC_Dalpha") || is(".LEPS_Dalpha")) {
      for (int k = 0; k < 9; k += 3) {
        c[k] = c[k] / kA0A;
        c[k + 1] = c[k + 1] * kA0A;
        c[k + 2] = c[k + 2] / eev;
      }
      l1041(1, c[0], c[1], c[2]);
      l1041(2, c[3], c[4], c[5]);
      l1041(3, c[6], c[7], c[8]);
      std::printf(" a = %s; b = %s; c = %s\n", fort_e(c[9], 10, 4).c_str(),
                  fort_e(c[10], 10, 4).c_str(), fort_e(c[11], 10, 4).c_str());
    } else if (is(".BARRIERXY_au") || is(".WELLXY_au")) {
      std::printf("%s", au);
      l1051i(1, c[0], c[1], c[2]);
      l1051i(2, c[3], c[4], c[5]);
    } else if (is(".BARRIERX_au") || is(".BARRIERY_au") || is(".WELLX_au") || is(".WELLY_au")) {
      std::printf("%s", au);
      l1051i(is(".BARRIERX") || is(".WELLX") ? 1 : 2, c[0], c[1], c[2]);
    } else if (is(".BARRIER_au") || is(".WELL_au")) {
      std::printf("%s", au);
      l1051i(1, c[0], c[1], c[4]);
      l1051i(2, c[2], c[3], c[4]);
    } else if (is(".CONST_au")) {
      std::printf("%s", au);
      l1061();
    } else if (is(".BARRIERXY") || is(".WELLXY")) {
      for (int k = 0; k < 6; k += 3) {
        c[k] = c[k] / kA0A;
        c[k + 1] = c[k + 1] / kA0A;
        c[k + 2] = c[k + 2] / eev;
      }
      l1051i(1, c[0], c[1], c[2]);
      l1051i(2, c[3], c[4], c[5]);
    } else if (is(".BARRIERX") || is(".BARRIERY") || is(".WELLX") || is(".WELLY")) {
      c[0] = c[0] / kA0A;
      c[1] = c[1] / kA0A;
      c[2] = c[2] / eev;
      l1051i(is(".BARRIERX") || is(".WELLX") ? 1 : 2, c[0], c[1], c[2]);
    } else if (is(".BARRIER") || is(".WELL")) {
      for (int k = 0; k < 4; ++k) c[k] = c[k] / kA0A;
      c[4] = c[4] / eev;
      l1051i(1, c[0], c[1], c[4]);
      l1051i(2, c[2], c[3], c[4]);
    } else if (is(".CONST") || is(".FREE")) {
      c[0] = c[0] / eev;
      l1061();
    } else {
      // makecst.f:337-339: the message, and the constants stay as read
      std::printf("%s", bad);
    }
    return;
  }
  if (is(".OHS")) {
    const double fk1 = sq(((c[1] * ccgs) * tau) * twopi) * sm1;
    c[0] = c[0] / kA0A;
    c[1] = fk1;
    l1031(1, c[0], c[1]);
  } else if (is(".DOHS")) {
    const double fk1 = sq(c[1] * ffreq) * sm1;
    const double fk2 = sq(((c[4] * ccgs) * tau) * twopi) * sm1 / sq(kA0A * 1.0e-10);
    const double re1 = c[0] / kA0A, re2 = c[2] / kA0A, re3 = c[3] / kA0A;
    c[0] = re1;
    c[1] = fk1;
    c[2] = re2;
    c[3] = re3;
    c[4] = fk2;
    l1031(1, c[0], c[1]);
    l1031(2, c[2], c[3]);
  } else if (is(".MORSE_Dalpha_au") || is(".ANTI-MORSE_Dalpha_au") || is(".MORSEM_Dalpha_au") ||
             is(".ANTI-MORSEM_Dalpha_au") || is(".MOD-MORSE_Dalpha_au")) {
    std::printf("%s", au);
    l1041(1, c[0], c[1], c[2]);
  } else if (is(".MORSE_Dalpha") || is(".ANTI-MORSE_Dalpha") || is(".MORSEM_Dalpha") ||
             is(".ANTI-MORSEM_Dalpha") || is(".MOD-MORSE_Dalpha")) {
    c[0] = c[0] / kA0A;
    c[1] = c[1] * kA0A;
    c[2] = c[2] / eev;
    l1041(1, c[0], c[1], c[2]);
  } else if (is(".MORSE") || is(".ANTI-MORSE") || is(".MORSEM") || is(".ANTI-MORSEM") ||
             is(".MOD-MORSE")) {  // the _CM^1 names share these prefixes
    const double re1 = c[0] / kA0A;
    const double fk1 = sq(((c[1] * ccgs) * tau) * twopi) * sm1;
    const double d1 = (((twopi * ccgs) * tau) * sq(c[1])) / (4.0 * c[2]);
    const double al1 = std::sqrt(fk1 / (2.0 * d1));
    c[0] = re1;
    c[1] = al1;
    c[2] = d1;
    l1041(1, c[0], c[1], c[2]);
  } else if (is(".BARRIER_au") || is(".WELL_au")) {
    std::printf("%s", au);
    l1051();
  } else if (is(".CONST_au")) {
    std::printf("%s", au);
    l1061();
  } else if (is(".BARRIER") || is(".WELL")) {
    c[0] = c[0] / kA0A;
    c[1] = c[1] / kA0A;
    c[2] = c[2] / eev;
    l1051();
  } else if (is(".CONST") || is(".FREE")) {
    c[0] = c[0] / eev;
    l1061();
  } else {
    std::printf("%s", bad);
    throw DeckError{"potential " + potch + ": no unit conversion for .1D (makecst.f:170-174)"};
  }
}

struct Run {
  int nd = 1, np[3] = {1, 1, 1};
  std::string dim = ".1D", potch = ".NULL", potchf = ".NULL", potfile, tpclc = ".SPECTRUM", tdi = ".NC";
  std::string inieigvc = ".CALC", prtcrl = ".NO", tppropg = ".NULL", tptrans = ".ONE";
  std::string tpabsor, tpwind = ".NONE";
  bool change = false, shiftp = true, absorb = false, fstop = true, lhwhm = false;
  double sm[3] = {1, 1, 1}, smf[3] = {1, 1, 1};
  double ti = 0.0, tf = 1e-4, dt = 1e-4, tol = 3.0, wp = 0.0;
  double chwhm = 0.0, de = 0.0, e1i = 0.0, ade = 0.0;
  double voi[3] = {0, 0, 0}, al[3] = {0, 0, 0}, ar[3] = {0, 0, 0};
  int mf = 13, mp = 10, prpgstate = 0;
  // *PULSE_AND_DIPOLE (rdinput.f:549-578; defaults espec.f:124-177)
  std::string efc = ".NONE", tpdipl = ".NULL", dmfile;
  double e0 = 0.0, tp = 0.0, omg = 0.0, t0 = 0.0, td = 0.0, sni = 0.0;
  int kl = 0, npr = 1, kp = 1;
  std::vector<double> cstdm;
  // analytic potential (rdinput.f:193-205: CSTI then CSTF records) and
  // *GRID_RANGES in angstrom (rdinput.f:206-214)
  std::vector<double> csti, cstf;
  double gxi[3] = {0, 0, 0}, gxf[3] = {0, 0, 0};
  // **TI (rdinput.f:370-381; defaults espec.f:129, 141-157): NIS states from
  // the IIL-th, counted from 0 as in the deck
  std::string tpdiag = ".MTRXDIAG";
  int nis = 1, iil = 0, nfs = 0, ifl = 0;  // *NIST; *NFST (the final states of .TI)
  double abstol = 1e-6;
  std::string fileaux;  // .ONLYSPEC: the output file holding a correlation function
  bool calc() const { return starts(inieigvc, ".CALC"); }
  bool onlyspec() const { return starts(tpclc, ".ONLYSPEC"); }
  bool energy() const { return starts(tpclc, ".ENERGY"); }
  bool pes() const { return starts(tpclc, ".PES") || starts(tpclc, ".POTENTIAL"); }
  bool collision() const { return starts(tpclc, ".COLLISION"); }
  double rk[3] = {0, 0, 0}, ra[3] = {0, 0, 0}, x0[3] = {0, 0, 0};  // .COLLISION wave packet
  bool prtpot = false;
  bool ti_form() const { return starts(tdi, ".TI"); }  // .ENERGY or .SPECTRUM .TI
};

const std::string& rec(const std::vector<std::string>* r, size_t i, const char* key) {
  if (!r || r->size() <= i) throw DeckError{std::string("missing record of ") + key};
  return (*r)[i];
}

bool yes_opt(const std::string& o) { return !(starts(o, ".NO") || starts(o, ".OFF")); }

// rdinput.f:125-620 for the keywords covered; print and output-file switches
// are accepted and not acted on
Run read_run(const Deck& d) {
  Run r;
  static const char* kIgnored[] = {"*TITLE", "*PRTEIGVC", "*PRTVEFF", "*PRTEIGVC2",
                                   "*PRTPULSE", "*PRTDIPOLE", "*PRTREGION", "*PRTONLYREIM"};
  auto ignored = [&](const std::string& k) {
    for (const char* x : kIgnored)
      if (k == x) return true;
    return false;
  };
  for (const auto& s : d.sec) {
    const std::string& sname = s.first;
    if (sname != "**MAIN" && sname != "**TI" && sname != "**TD" && sname != "**SPECTRUM" &&
        sname != "**END")
      throw DeckError{"section " + sname + " is not covered (collision runs are not)"};
    for (const auto& kv : s.second) {
      const std::string& k = kv.first;
      const std::vector<std::string>* v = &kv.second;
      if (ignored(k)) continue;
      if (sname == "**MAIN") {
        if (k == "*DIMENSION") {
          r.dim = upper(rec(v, 0, "*DIMENSION"));
          if (starts(r.dim, ".1D") && !starts(r.dim, ".1DC")) r.nd = 1;
          else if (r.dim.size() >= 3 && starts(r.dim, ".2D") && (r.dim.size() == 3 || r.dim[3] == ' ')) r.nd = 2;
          else if (starts(r.dim, ".3D")) r.nd = 3;
          else throw DeckError{"*DIMENSION " + r.dim + " is not covered (.1D, .2D, .3D)"};
          const std::vector<double> n = numbers(rec(v, 1, "*DIMENSION"));
          if ((int)n.size() < r.nd) throw DeckError{"*DIMENSION: grid sizes missing"};
          for (int a = 0; a < r.nd; ++a) r.np[a] = (int)n[a];
        } else if (k == "*POTENTIAL") {
          // the names are compared as written (makecst.f: '.MORSE_Dalpha_au', ...)
          r.potch = r.potchf = rec(v, 0, "*POTENTIAL");
          if (starts(r.potch, ".FILE")) {
            r.potfile = rec(v, 1, "*POTENTIAL");
          } else {
            r.csti = numbers(rec(v, 1, "*POTENTIAL"));
            r.cstf = numbers(rec(v, 2, "*POTENTIAL"));
          }
        } else if (k == "*INITIAL_POTENTIAL" || k == "*FINAL_POTENTIAL") {
          // rdinput.f:177-191: one surface with its one constant record
          const bool ini = k == "*INITIAL_POTENTIAL";
          (ini ? r.potch : r.potchf) = rec(v, 0, k.c_str());
          if (starts(ini ? r.potch : r.potchf, ".FILE"))
            throw DeckError{k + " .FILE: a .FILE potential is read with *POTENTIAL"};
          (ini ? r.csti : r.cstf) = numbers(rec(v, 1, k.c_str()));
        } else if (k == "*GRID_RANGES") {
          const std::vector<double> x = numbers(rec(v, 0, "*GRID_RANGES"));
          // rdinput.f:206-214: columns 14-15 'au' give bohr
          const std::string& h = d.head.at(sname).at(k);
          const bool au = h.size() >= 15 && h.compare(13, 2, "au") == 0;
          for (size_t a = 0; a < 3 && 2 * a + 1 < x.size(); ++a) {
            r.gxi[a] = au ? x[2 * a] * kA0A : x[2 * a];
            r.gxf[a] = au ? x[2 * a + 1] * kA0A : x[2 * a + 1];
          }
        } else if (k == "*MASS") {
          const std::vector<double> m = numbers(rec(v, 0, "*MASS"));
          for (size_t a = 0; a < m.size() && a < 3; ++a) r.sm[a] = m[a];
        } else if (k == "*MASS_FACTOR") {
          const std::vector<double> m = numbers(rec(v, 0, "*MASS_FACTOR"));
          for (size_t a = 0; a < m.size() && a < 3; ++a) r.smf[a] = m[a];
        } else if (k == "*TPCALC") {
          r.tpclc = upper(rec(v, 0, "*TPCALC"));
          if (starts(r.tpclc, ".SPECTRUM")) r.tdi = upper(rec(v, 1, "*TPCALC"));
          else if (starts(r.tpclc, ".PROPAGATION") || starts(r.tpclc, ".CORRELATION") ||
                   starts(r.tpclc, ".COLLISION"))
            r.tdi = ".TD";
          else if (starts(r.tpclc, ".ONLYSPEC")) r.fileaux = rec(v, 1, "*TPCALC");  // TDI .NC
          else if (starts(r.tpclc, ".ENERGY")) r.tdi = ".TI";
          else if (starts(r.tpclc, ".PES") || starts(r.tpclc, ".POTENTIAL")) r.tdi = ".NC";
          else throw DeckError{"*TPCALC " + r.tpclc + " is not covered"};
        } else if (k == "*INIEIGVC") {
          r.inieigvc = upper(rec(v, 0, "*INIEIGVC"));
        } else if (k == "*CHANGE") {
          r.change = yes_opt(upper(rec(v, 0, "*CHANGE")));
        } else if (k == "*SHIFT_POTENTIAL") {
          r.shiftp = yes_opt(upper(rec(v, 0, "*SHIFT_POTENTIAL")));
        } else if (k == "*PRTPOT") {  // rdinput.f:289-296
          const std::string o = upper(rec(v, 0, "*PRTPOT"));
          r.prtpot = starts(o, ".YES") || starts(o, ".ON");
        } else if (k == "*DONOTSTOP") {
          r.fstop = !yes_opt(upper(rec(v, 0, "*DONOTSTOP")));
        } else if (k == "*PRTCRL") {
          std::string p = upper(rec(v, 0, "*PRTCRL"));
          if (starts(p, ".FULL") || starts(p, ".ALL")) p = ".YES";  // rdinput.f:332-338
          if (starts(p, ".NONE") || starts(p, ".NULL") || starts(p, ".EMPTY")) p = ".NO";
          r.prtcrl = p;
        } else {
          throw DeckError{"keyword " + k + " of **MAIN is not covered"};
        }
      } else if (sname == "**TI") {
        // rdinput.f:355-381: an initial potential of its own, the
        // diagonalisation and the states it keeps
        if (k == "*INITIAL_POTENTIAL" || k == "*INITIAL_CONDITION" || k == "*INITIAL_WP" ||
            k == "*INITIAL_WF" || k == "*INITIAL_WAVE_FUNCTION" || k == "*WAVE_FUNCTION" ||
            k == "*WAVE_PACKET" || k == "*POTENTIAL") {
          r.potch = rec(v, 0, k.c_str());
          if (starts(r.potch, ".FILE")) r.potfile = rec(v, 1, k.c_str());
          else r.csti = numbers(rec(v, 1, k.c_str()));
        } else if (k == "*TPDIAG") {
          r.tpdiag = upper(rec(v, 0, "*TPDIAG"));
        } else if (k == "*NIST") {
          const std::vector<double> x = numbers(rec(v, 0, "*NIST"));
          if (x.size() < 2) throw DeckError{"*NIST: NIS IIL"};
          r.nis = (int)x[0];
          r.iil = (int)x[1];
        } else if (k == "*ABSTOL") {
          r.abstol = numbers(rec(v, 0, "*ABSTOL")).at(0);
        } else if (k == "*NFST") {
          const std::vector<double> x = numbers(rec(v, 0, "*NFST"));
          if (x.size() < 2) throw DeckError{"*NFST: NFS IFL"};
          r.nfs = (int)x[0];
          r.ifl = (int)x[1];
        } else if (k == "*COLLISION_ENERGY" || k == "*SIZE_OF_GAUSSIAN" ||
                   k == "*INIT_POSSITION") {
          // rdinput.f:384-419: per axis; the energy in eV unless columns 19-20
          // read 'au', the size multiplied by A0A when they do, the position
          // as written
          const std::vector<double> x = numbers(rec(v, 0, k.c_str()));
          const std::string& h = d.head.at(sname).at(k);
          const bool au = h.size() >= 20 && h.compare(18, 2, "au") == 0;
          for (size_t a = 0; a < 3 && a < x.size(); ++a) {
            if (k == "*COLLISION_ENERGY") r.rk[a] = au ? x[a] : x[a] / 27.2113834;
            else if (k == "*SIZE_OF_GAUSSIAN") r.ra[a] = au ? x[a] * kA0A : x[a];
            else r.x0[a] = x[a];
          }
        } else if (k == "*SEED" || k == "*MAXINT") {
          continue;  // the seed and the length of LANCZSG's iterations
        } else {
          throw DeckError{"keyword " + k + " of **TI is not covered"};
        }
      } else if (sname == "**TD") {
        if (k == "*PROPAG") {
          r.tppropg = upper(rec(v, 0, "*PROPAG"));
          const std::string& line = rec(v, 1, "*PROPAG");
          const std::vector<double> x = numbers(line);
          const bool sil = starts(r.tppropg, ".PSIL") || starts(r.tppropg, ".PPSIL") ||
                           starts(r.tppropg, ".PPLNZ");  // rdinput.f:439-444
          // a '/' ends the list early and leaves MP at its default
          const bool slash = line.find('/') != std::string::npos;
          if (x.size() < (sil && !slash ? 4u : 3u))
            throw DeckError{"*PROPAG: TI TF DT" + std::string(sil ? " MP" : "")};
          r.ti = x[0];
          r.tf = x[1];
          r.dt = x[2];
          if (!(r.dt > 0.0) || !((r.tf - r.ti) / r.dt < 1.0e9))
            throw DeckError{"*PROPAG: DT must be positive and (TF - TI)/DT below 1e9"};
          if (sil && x.size() >= 4) r.mp = (int)x[3];
        } else if (k == "*PRPGSTATE") {
          r.prpgstate = (int)numbers(rec(v, 0, "*PRPGSTATE")).at(0);
        } else if (k == "*TPTRANS") {
          r.tptrans = upper(rec(v, 0, "*TPTRANS"));
        } else if (k == "*PRPTOL") {
          r.tol = numbers(rec(v, 0, "*PRPTOL")).at(0);
        } else if (k == "*NSHOT") {
          continue;  // the snapshot period of the files PPSOD writes
        } else if (k == "*NPROJECTIONS") {
          const std::vector<double> x = numbers(rec(v, 0, "*NPROJECTIONS"));
          if (x.size() < 2) throw DeckError{"*NPROJECTIONS: NPR KP"};
          r.npr = (int)x[0];
          r.kp = (int)x[1];
        } else if (k == "*PULSE_AND_DIPOLE") {
          r.efc = upper(rec(v, 0, "*PULSE_AND_DIPOLE"));
          size_t i = 1;
          const bool gaus = starts(r.efc, ".GAUS"), ggaus = starts(r.efc, ".GGAUS");
          const bool sin2 = starts(r.efc, ".SIN2"), none = starts(r.efc, ".NONE");
          if (!gaus && !ggaus && !sin2 && !none)
            throw DeckError{"*PULSE_AND_DIPOLE " + r.efc + ": the pulse is not known (ef.f:44-60)"};
          const std::vector<double> x = numbers(rec(v, i++, "*PULSE_AND_DIPOLE"));
          if (!none) {
            if (x.size() < (ggaus ? 6u : 5u))
              throw DeckError{"*PULSE_AND_DIPOLE: E0 TP OMG " + std::string(sin2 ? "TD" : "T0") +
                              " SNI" + (ggaus ? " KL" : "")};
            r.e0 = x[0];
            r.tp = x[1];
            r.omg = x[2];
            (sin2 ? r.td : r.t0) = x[3];
            r.sni = x[4];
            if (ggaus) r.kl = (int)x[5];
          }
          r.tpdipl = upper(rec(v, i++, "*PULSE_AND_DIPOLE"));
          if (starts(r.tpdipl, ".READ") || starts(r.tpdipl, ".GET")) {
            r.dmfile = rec(v, i++, "*PULSE_AND_DIPOLE");  // rdinput.f:571-572
            if (starts(r.tpdipl, ".GET"))
              throw DeckError{"desired dipole moment .GET wasn't found (dipl.f:86-89)"};
          } else if (!starts(r.tpdipl, ".NULL")) {
            if (!starts(r.tpdipl, ".CONST") && !starts(r.tpdipl, ".EXP") &&
                !starts(r.tpdipl, ".NONE"))
              throw DeckError{"desired dipole moment " + r.tpdipl + " wasn't found (dipl.f:86-89)"};
            r.cstdm = numbers(rec(v, i++, "*PULSE_AND_DIPOLE"));
            if (r.cstdm.size() < (starts(r.tpdipl, ".EXP") ? 2u : 1u))
              throw DeckError{"*PULSE_AND_DIPOLE: dipole constants missing"};
          }
        } else if (k == "*ABSORBING") {
          r.tpabsor = rec(v, 0, "*ABSORBING");  // '.SMOOTHW_au' as written
          if (starts(r.tpabsor, ".NULL")) continue;
          if (!starts(r.tpabsor, ".SMOOTHW") && !starts(r.tpabsor, ".SMRS") &&
              !starts(r.tpabsor, ".VOPTIC"))
            throw DeckError{"*ABSORBING " + r.tpabsor + " is not known (rdinput.f:526-548)"};
          r.absorb = true;
          const std::vector<double> vo = numbers(rec(v, 1, "*ABSORBING"));
          const std::vector<double> lr = numbers(rec(v, 2, "*ABSORBING"));
          for (size_t a = 0; a < 3 && a < vo.size(); ++a) r.voi[a] = vo[a];
          for (size_t a = 0; a < 3 && 2 * a + 1 < lr.size(); ++a) {
            r.al[a] = lr[2 * a];
            r.ar[a] = lr[2 * a + 1];
          }
        } else {
          throw DeckError{"keyword " + k + " of **TD is not covered"};
        }
      } else if (sname == "**SPECTRUM") {
        if (k == "*FOURIER") {
          r.mf = (int)numbers(rec(v, 0, "*FOURIER")).at(0);
        } else if (k == "*WINDOWING") {
          r.tpwind = upper(rec(v, 0, "*WINDOWING"));
          r.wp = numbers(rec(v, 1, "*WINDOWING")).at(0);
        } else if (k == "*HWHM") {
          const std::vector<double> h = numbers(rec(v, 0, "*HWHM"));
          if (h.size() < 4) throw DeckError{"*HWHM: CHWHM DE E1I ADE"};
          r.chwhm = h[0];
          r.de = h[1];
          r.e1i = h[2];
          r.ade = h[3];
          r.lhwhm = true;
        } else {
          throw DeckError{"keyword " + k + " of **SPECTRUM is not covered"};
        }
      }
    }
  }
  if (r.onlyspec()) return r;  // no grid, potential or propagation (espec.f:602)
  if (r.pes()) {  // espec.f:860-881: the initial potential only
    if (starts(r.potch, ".FILE") || starts(r.potch, ".NULL"))
      throw DeckError{"*TPCALC .PES: an analytic initial potential is covered"};
    if (r.nd > 2) throw DeckError{"*TPCALC .PES: .1D and .2D grids are covered"};
    for (int a = 0; a < r.nd; ++a)
      if (!(r.gxf[a] > r.gxi[a])) throw DeckError{"*GRID_RANGES: XI < XF is needed"};
    return r;
  }
  const bool file_i = starts(r.potch, ".FILE"), file_f = starts(r.potchf, ".FILE");
  if (starts(r.potch, ".NULL") || starts(r.potchf, ".NULL"))
    throw DeckError{"*POTENTIAL is missing"};
  // espec.f:410-413: an analytic potential always has its state computed
  if (!file_i && !r.calc()) {
    std::printf(" -> Warning! Replacing *INIEIGVC to .CALC\n");
    r.inieigvc = ".CALC";
  }
  if (file_i != file_f)
    throw DeckError{"an initial potential from a .FILE with an analytic final one (or the "
                    "reverse) is not covered"};
  if (file_i && !starts(r.inieigvc, ".GETR") && !starts(r.inieigvc, ".READR"))
    throw DeckError{"*INIEIGVC " + r.inieigvc + ": a .FILE potential is covered with .GETR (the "
                    "eigenvector of the .FILE)"};
  if (!starts(r.tptrans, ".ONE"))
    throw DeckError{"one propagated state (*TPTRANS .ONE) is covered"};
  if (r.collision()) {
    // espec.f:849-864 with init_cond.f:18-38: a Gaussian wave packet with a
    // momentum on an analytic .1D potential (the .2D forms build on a .FILE
    // eigenvector, .GETR2/.GETC*)
    if (r.nd != 1 || file_i || !r.calc())
      throw DeckError{".COLLISION: the .1D wave packet of an analytic potential is covered "
                      "(*INIEIGVC .CALC)"};
    if (!(r.gxf[0] > r.gxi[0])) throw DeckError{"*GRID_RANGES: XI < XF is needed"};
    if (!(r.ra[0] > 0.0)) throw DeckError{"*SIZE_OF_GAUSSIAN must be positive"};
  } else if (r.calc()) {
    if (r.nd > 2)
      throw DeckError{"computed initial states (.CALC) are covered on .1D and .2D grids (the "
                      "GPU eigensolver's)"};
    for (int a = 0; a < r.nd; ++a)
      if (!(r.gxf[a] > r.gxi[a])) throw DeckError{"*GRID_RANGES: XI < XF is needed"};
    // espec.f:1083: the propagated state is column NISPG - IIL + 1 of the NIS
    // computed ones (IIL, NISPG counted from 1 there)
    if (r.nis < 1 || r.iil < 0 ||
        (!r.ti_form() && (r.prpgstate < r.iil || r.prpgstate >= r.iil + r.nis)))
      throw DeckError{"*PRPGSTATE must be one of the states *NIST computes"};
    if (r.iil + r.nis > 16 || r.prpgstate >= 16 || r.ifl + r.nfs > 16)
      throw DeckError{"*NIST, *NFST: the GPU eigensolver computes the 16 lowest states at most"};
    if (r.ti_form() && !r.energy() && (r.nfs < 1 || r.ifl < 0))
      throw DeckError{"*NFST: the .TI spectrum needs final states"};
    if (!starts(r.tpdiag, ".MTRXDIAG") && !starts(r.tpdiag, ".LANCZS"))
      throw DeckError{"*TPDIAG " + r.tpdiag + ": initial eigenvalue(s) and eigenvector(s) "
                      "error (espec.f:920-925)"};
  } else if (r.prpgstate != 0) {
    throw DeckError{".GETR gives one state: *PRPGSTATE 0"};
  }
  if (starts(r.tpdipl, ".EXP+") && !r.calc())
    throw DeckError{"dipole .EXP+ is normalised at the final potential's Re (CSTF(1), dipl.f), "
                    "which a .FILE potential leaves at zero"};
  if (starts(r.tpclc, ".SPECTRUM") && !starts(r.tdi, ".TD") && !starts(r.tdi, ".TI"))
    throw DeckError{"*TPCALC .SPECTRUM " + r.tdi + ": .TD and .TI are covered"};
  if (r.ti_form()) {
    if (!r.calc()) throw DeckError{"the .TI formalism computes the states: *INIEIGVC .CALC"};
    return r;  // no propagation
  }
  if (!starts(r.tppropg, ".PFSPO") && !starts(r.tppropg, ".PFSOD") &&
      !starts(r.tppropg, ".PSIL") && !starts(r.tppropg, ".PSOD") && !starts(r.tppropg, ".PPSOD") &&
      !starts(r.tppropg, ".PPSIL") && !starts(r.tppropg, ".PPLNZ"))
    throw DeckError{"propagator " + r.tppropg + " is not covered (.PFSPO, .PFSOD, .PSIL, .PSOD, "
                    ".PPSOD, .PPSIL, .PPLNZ)"};
  // rdinput.f:650-660 with NIS = 1 for .GETR.  The populations PPSOD prints
  // are on LNZVC(., KP+1..KP+NPR), PPLNZ's on LNZVC(., KP+1..KP+NPR-1): the
  // eigenvector matrix, which holds the NIS computed states for .CALC; for
  // .GETR the executable holds its column 1 at zero at the call
  const int nis = r.calc() ? r.nis : 1;
  if (r.npr + r.kp > nis) r.npr -= nis;
  if (r.npr > 6) r.npr = 6;
  const int printed_w = starts(r.tppropg, ".PPSOD") ? r.npr
                        : (starts(r.tppropg, ".PPSIL") || starts(r.tppropg, ".PPLNZ")) ? r.npr - 1
                                                                                        : 0;
  if (printed_w > 0 && !r.calc() && (r.kp != 0 || printed_w > 1))
    throw DeckError{"*NPROJECTIONS: projections on computed eigenstates need .CALC (.GETR "
                    "gives one state; KP = 0 with one printed projection is covered)"};
  if (printed_w > 0 && r.calc() && (r.kp < 0 || r.kp + printed_w > r.nis))
    throw DeckError{"*NPROJECTIONS: the projections reach past the states *NIST computes"};
  return r;
}

Run load_run(const std::string& deck_path) {
  std::ifstream in(deck_path);
  if (!in) throw DeckError{"cannot open " + deck_path};
  std::stringstream ss;
  ss << in.rdbuf();
  return read_run(parse_deck(ss.str()));
}

// C(t) stride NC and the final time (espec.f:1328-1353); prints the
// reference's warning when TF changes
int c_stride(Run& r) {
  int nc = 0;
  for (;;) {
    const double sc = 2.0 * (r.tf - r.ti) / r.dt;
    nc = (int)(sc / std::pow(2.0, r.mf));
    if (std::fabs(sc - nc * std::pow(2.0, r.mf)) >= 1e-10 && r.change) {
      r.tf = nc * std::pow(2.0, r.mf - 1.0) * r.dt;
      std::printf(" -> Warning! Final time changed to%s\n", list_real(r.tf).c_str());
      continue;
    }
    if (std::fabs(sc - nc * std::pow(2.0, r.mf)) >= 1e-10 && starts(r.tpclc, ".SPECTRUM")) {
      std::printf(" <<<>>> Final time is not adequate for FFT <<<>>>\n");
      if (r.fstop) throw DeckError{"final time is not adequate for FFT"};
    }
    break;
  }
  if (nc < 1) throw DeckError{"the C(t) stride is below one step: raise TF or lower MF"};
  return nc;
}

// total correlation (espec.f:1545-1576): C(-t) = C(t)*, 2^MF samples from the
// first MC = 2^(MF-1) recorded C values
void total_correlation(int mc, const double* cr, const double* ci, std::vector<double>& cu,
                       std::vector<double>& cv) {
  cu.assign(2 * (size_t)mc, 0.0);
  cv.assign(2 * (size_t)mc, 0.0);
  for (int i = 1; i <= mc; ++i) {
    cu[mc + i - 1] += cr[i - 1];
    cu[mc - i + 1] = cu[mc + i - 1];
    cv[mc + i - 1] += ci[i - 1];
    cv[mc - i + 1] = -cv[mc + i - 1];
  }
  cu[0] += cr[mc - 1];
  cv[0] += ci[mc - 1];
  cv[0] = -cv[0];
}

// the "Correlation Function:" block (FORMAT 1041 / 1042)
std::string correlation_table(int mc, double tf, const std::vector<double>& cu,
                              const std::vector<double>& cv, double dtf = 0.0) {
  std::string out = " \n Correlation Function:\n \"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\n";
  out += "       *t/fs*       *C(t)r*       *C(t)i*\n";
  if (dtf == 0.0) dtf = tf / mc;  // espec.f:1548 (GETCORR's DTF for .ONLYSPEC)
  char buf[128];
  for (int i = 1; i <= 2 * mc; ++i) {
    const double t = -tf + (i - 1.0) * dtf;
    std::snprintf(buf, sizeof buf, "%15.6f   %10.7f    %10.7f\n", t, cu[i - 1], cv[i - 1]);
    out += buf;
  }
  return out;
}

// PRTPT (prtpot.f:1-47) on standard output: the FORMAT 1011 header and one
// FORMAT 1012 row per grid point (coordinates last axis first, |V| < 1e-99
// printed as zero); gfortran ends each record at its last item
void prtpt(int nd, const int* np, const double* xi, const double* sh, const double* v) {
  std::string out = "    ";
  for (int a = nd; a >= 1; --a) out += " *R" + std::to_string(a) + "*" + std::string(10, ' ');
  out += " *V0*\n";
  const int n1 = np[0], n2 = nd > 1 ? np[1] : 1, n3 = nd > 2 ? np[2] : 1;
  for (int l = 0; l < n3; ++l)
    for (int k = 0; k < n2; ++k)
      for (int j = 0; j < n1; ++j) {
        const double xp[3] = {xi[0] + j * sh[0], xi[1] + k * sh[1], xi[2] + l * sh[2]};
        const double w = v[j + (size_t)n1 * (k + (size_t)n2 * l)];
        out += " ";
        for (int a = nd - 1; a >= 0; --a) out += fort_e(xp[a], 12, 6) + "   ";
        out += fort_e(std::fabs(w) < 1e-99 ? 0.0 : w, 12, 6) + "\n";
      }
  std::fwrite(out.data(), 1, out.size(), stdout);
}

// Device buffers of one deck run, freed on every exit
struct DevBufs {
  std::vector<void*> p;
  double* alloc(size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(double) * (count ? count : 1)) != cudaSuccess)
      throw DeckError{"device memory for the initial state"};
    p.push_back(q);
    return (double*)q;
  }
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
};

// The time-independent part of espec.f for an analytic .1D or .2D potential: the
// grid of *GRID_RANGES in bohr (espec.f:345, 618-641), MAKECST of both constant
// records (espec.f:683-690), GVPOT of the initial potential (espec.f:865-869),
// its eigenstates IIL..IIU (espec.f:872-927) and GVPOT of the final potential
// (espec.f:985-990), both potentials on the GPU.  MTRXDIAG (DSPEVX of the
// packed AP1D matrix) and LANCZS both diagonalise the finite-difference
// Hamiltonian of AP1D / AU1D; here the GPU eigensolver does, its states
// converged to a residual of 1e-12 ||H|| (the reference's ABSTOL = 1e-6 bounds
// only the bisection of its eigenvalues).  Returns the propagated state
// (EIGVC(., K), espec.f:1262-1265) and the final potential; eigvc: the NIS
// states, n each; r.e1i = E1I (espec.f:927).
FileData initial_state(Run& r, double* sh, double* shm, double* sm, std::vector<double>& eigvc) {
  const int nd = r.nd;
  int n = 1;
  FileData fd;
  for (int a = 0; a < nd; ++a) {
    n *= r.np[a];
    sm[a] = kAmu * r.sm[a];
    sh[a] = ((r.gxf[a] - r.gxi[a]) / (r.np[a] - 1.0)) / kA0A;
    fd.xi[a] = r.gxi[a] / kA0A;
    fd.xf[a] = r.gxf[a] / kA0A;
    shm[a] = 1.0 / ((((24.0 * sm[a]) * r.smf[a]) * sh[a]) * sh[a]);  // espec.f:630
  }
  // espec.f:252-258, 613-616: a third mass (in atomic units) for the
  // mass-scaled coordinates of .LEPS_CC on a .2D grid
  const bool cc = nd == 2 && (starts(r.potch, ".LEPS_CC") || starts(r.potchf, ".LEPS_CC"));
  sm[2] = cc ? kAmu * r.sm[2] : r.sm[2];
  // espec.f:683-690: a surface named .NULL (a .PES deck's final one) is not converted
  const bool final_surface = !starts(r.potchf, ".NULL");
  std::printf(" Initial potential:\n");
  makecst(nd, r.potch, sm, r.csti);
  if (final_surface) {
    std::printf(" Final potential:\n");
    makecst(nd, r.potchf, sm, r.cstf);
  }
  std::printf(" \n Units converted.\n");
  const int ki = espec_pot_kind(r.potch.c_str(), r.potch.size(), nd);
  const int kf = final_surface ? espec_pot_kind(r.potchf.c_str(), r.potchf.size(), nd) : -1;
  if (!ki || !kf)
    throw DeckError{"potential " + (ki ? r.potchf : r.potch) + " is not a form of " + r.dim +
                    " grids (potfuncs.f)"};
  if (r.collision()) {
    // espec.f:849-864: the wave packet instead of eigenstates, then the
    // final surface; INIT_COND (init_cond.f:18-38) and GET_GAUSS (gauss.f:20):
    // psi = N exp(-ln2 ((x - X0)/A)^2) e^{i k (x - X0)}, k = +-sqrt(2 m |E|)
    msg1003("Computing the initial wave packet...");
    double rk = r.rk[0];
    rk = rk < 0.0 ? -std::sqrt(-(((2.0 * sm[0]) * r.smf[0]) * rk))
                  : std::sqrt(((2.0 * sm[0]) * r.smf[0]) * rk);
    const double ln2 = 0.69314718;  // gauss.f's constant as written
    auto gauss = [&](double coord, double norm) {
      const double q = coord / r.ra[0];
      return norm * std::exp(-ln2 * (q * q));
    };
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) {
      const double g = gauss(fd.xi[0] + i * sh[0] - r.x0[0], 1.0);
      nrm = nrm + g * g;
    }
    nrm = 1.0 / std::sqrt(nrm);
    fd.psi.resize(n);
    fd.psi_im.resize(n);
    for (int i = 0; i < n; ++i) {
      const double coord = fd.xi[0] + i * sh[0] - r.x0[0];
      const double g = gauss(coord, nrm);
      fd.psi[i] = std::cos(rk * coord) * g;
      fd.psi_im[i] = std::sin(rk * coord) * g;
    }
    std::printf(" Initial wave packet computed.\n \n");
    DevBufs dev;
    double* d_vf = dev.alloc(n);
    double xmin = 0.0;
    msg1003("   Generating final potential...");
    fd.vpot.resize(n);
    if (espec_gvpot_1d(1, &n, fd.xi, sh, kf, r.cstf.data(), r.shiftp ? 1 : 0, d_vf, &xmin,
                       nullptr) ||
        cudaMemcpy(fd.vpot.data(), d_vf, sizeof(double) * n, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      throw DeckError{std::string("GVPOT: ") + espec_last_error()};
    std::printf(" Final potential generated.\n");
    std::printf("\n%33sStarting 0th state to be propagated...\n%12d th state started.\n", "", 0);
    eigvc.clear();
    return fd;
  }
  // espec.f:879-905: *CHANGE on a grid above 3e4 points switches to LANCZSG,
  // which keeps the ground state only
  std::string tpdiag = r.tpdiag;
  int iil = r.iil, nis = r.nis;
  const bool to_lanczsg = r.change && n > 30000;
  if (to_lanczsg) tpdiag = ".LANCZSG";
  const bool lanczsg = r.change && starts(tpdiag, ".LANCZSG");
  if (lanczsg) {
    iil = 0;
    nis = 1;
    if (r.prpgstate != 0 && !r.pes())
      throw DeckError{".LANCZSG keeps the ground state: *PRPGSTATE 0"};
  }
  const int nst = std::max(iil + nis, r.ti_form() ? 1 : r.prpgstate + 1);  // states 0 .. nst-1
  const int nstf = r.ti_form() ? r.ifl + r.nfs : 0;  // final states of .TI
  const int nbuf = std::max(nst, nstf);
  const int m = std::min(40, n);
  if (m < 2) throw DeckError{"the grid needs two points at least"};
  DevBufs dev;
  double* d_vi = dev.alloc(n);
  double* d_vf = dev.alloc(n);
  double* d_start = dev.alloc((size_t)nbuf * n);
  double* d_vec = dev.alloc((size_t)nbuf * n);
  double* d_eval = dev.alloc(nbuf);
  double* d_resid = dev.alloc(nbuf);
  int* d_mv = (int*)dev.alloc(nbuf);
  double* d_L = dev.alloc((size_t)m * n);
  double* d_w = dev.alloc(n);
  double xmin = 0.0, xminb = 0.0;
  // GVPOT (gvpot.f:21-64): XMIN is set for .1D grids only
  auto gvpot = [&](int kind, const double* cst, double* d_v, double* xm) {
    return nd == 1 ? espec_gvpot_1d(1, &n, fd.xi, sh, kind, cst, r.shiftp ? 1 : 0, d_v, xm,
                                    nullptr)
                   : espec_gvpot_nd(nd, r.np, fd.xi, sh, sm, kind, cst, r.shiftp ? 1 : 0, 0,
                                    d_v, nullptr);
  };
  // the lowest ns states of the potential on the device, to a residual of
  // 1e-12 ||H||; false if one did not converge
  const int npp[2] = {r.np[0], nd == 2 ? r.np[1] : 1};
  const double shmp[2] = {shm[0], nd == 2 ? shm[1] : 0.0};
  auto solve = [&](const double* d_v, int ns, std::vector<double>& ev, std::vector<double>& vec) {
    std::vector<double> v(n), resid(ns);
    if (cudaMemcpy(v.data(), d_v, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw DeckError{"copy of a potential"};
    double vmax = 0.0;
    for (double x : v) vmax = std::max(vmax, std::fabs(x));
    const double tol = 1e-12 * std::max(1.0, 64.0 * (shm[0] + shm[1]) + vmax);
    ev.assign(ns, 0.0);
    vec.assign((size_t)ns * n, 0.0);
    if (espec_eig_lcg_start(d_start, n, ns, nullptr) ||
        espec_eig_solve_dev(1, npp, shmp, d_v, d_start, ns, m, tol, 20000, d_vec, d_eval,
                            d_resid, d_mv, d_L, d_w, nullptr) ||
        cudaMemcpy(ev.data(), d_eval, sizeof(double) * ns, cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaMemcpy(resid.data(), d_resid, sizeof(double) * ns, cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaMemcpy(vec.data(), d_vec, sizeof(double) * ns * n, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      throw DeckError{std::string("eigenstates: ") + espec_last_error()};
    bool ok = true;
    for (int j = 0; j < ns; ++j) ok = ok && resid[j] <= tol;
    return ok;
  };
  // FORMAT 1014/1015 rows of states j0 .. j0+cnt-1
  auto table = [&](const std::vector<double>& ev, int j0, int cnt) {
    for (int j = j0; j < j0 + cnt; ++j)
      std::printf(" |   %3d        |  %s  |\n ---------------------------------\n", j,
                  fort_e(ev[j], 12, 6).c_str());
  };
  msg1003("Generating initial potential...");
  if (gvpot(ki, r.csti.data(), d_vi, &xmin))
    throw DeckError{std::string("GVPOT: ") + espec_last_error()};
  std::printf(" Initial potential generated.\n");
  if (r.prtpot || r.pes()) {
    std::vector<double> v(n);
    if (cudaMemcpy(v.data(), d_vi, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw DeckError{"copy of the initial potential"};
    if (r.prtpot) {  // espec.f:871-876
      std::printf(" \n Initial potential points:\n \"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\n");
      prtpt(nd, r.np, fd.xi, sh, v.data());
    }
    if (r.pes()) {  // espec.f:880-881
      fd.vpot = v;
      eigvc.clear();
      return fd;
    }
  }
  msg1003("Calculating eigenvalue(s) and eigenvector(s)");
  std::printf("   %68s\n", "for the initial state...");
  if (to_lanczsg) std::printf(" -> Type of diagonalization changed to: LANCZSG\n");
  if (lanczsg)
    std::printf(" -> .LANCZSG allows only the ground state eigenvectors calculation\n"
                " -> Total number of eigenvectors changed to %11d\n", 1);
  std::printf(" %s\n", starts(tpdiag, ".MTRXDIAG")   ? "Using complete matrix diagonalization procedure,"
                       : starts(tpdiag, ".LANCZSG") ? "Using interative lanczos tri-diagonalization procedure,"
                                                    : "Using lanczos tri-diagonalization procedure,");
  std::fflush(stdout);
  std::vector<double> eval;
  if (solve(d_vi, nst, eval, eigvc)) {
    std::printf(" \n Eigenvalues:\n \"\"\"\"\"\"\"\"\"\"\"\"\n");
    std::printf(" ---------------------------------\n");
    std::printf(" |  Eigenstate  |  Eigenvalues   |\n =================================\n");
    table(eval, iil, nis);
  } else {
    std::printf(" <<<>>> It wasn`t possible obtain eignvalues and eignvectors correctly <<<>>>\n"
                " Exiting.\n");
    if (r.fstop) throw DeckError{"the initial eigenstates did not converge"};
  }
  if (!r.ti_form()) r.e1i = eval[r.prpgstate] * 27.2113834;
  if (r.energy()) {  // espec.f:954: the eigenvalues only
    eigvc.clear();
    return fd;
  }
  std::printf(" \n");
  msg1003("   Generating final potential...");
  fd.vpot.resize(n);
  if (gvpot(kf, r.cstf.data(), d_vf, &xminb) ||
      cudaMemcpy(fd.vpot.data(), d_vf, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    throw DeckError{std::string("GVPOT: ") + espec_last_error()};
  if (std::fabs(xminb - xmin) < 1e-6)
    std::printf(" -> Warning: The initial and final potential have the same minimum possition.\n");
  std::printf(" Final potential generated.\n");
  if (r.prtpot) {  // espec.f:994-1010
    std::printf(" \n Final potential values:\n \"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\"\n");
    prtpt(nd, r.np, fd.xi, sh, fd.vpot.data());
  }
  if (r.ti_form()) {
    // espec.f:1015-1078: the final surface's states IFL..IFU and SPECTRUMTI
    msg1003("   Calculating eigenvalue(s) and eigenvector(s)");
    std::printf("   %68s\n", "      from final state...");
    std::printf(" %s\n", starts(tpdiag, ".MTRXDIAG")
                             ? "Using complete matrix diagonalization procedure."
                             : "Using lanczos tri-diagonalization procedure.");
    std::fflush(stdout);
    std::vector<double> evf, vecf;
    if (solve(d_vf, nstf, evf, vecf)) {
      std::printf(" \n Eigenvalues:\n \"\"\"\"\"\"\"\"\"\"\"\"\n");
      std::printf(" ---------------------------------\n");
      std::printf(" |  Eigenstate  |   Eigenvalues   |\n ==================================\n");
      table(evf, r.ifl, r.nfs);
    } else {
      std::printf(" <<<>>> It wasn`t able obtain eignvalues and eignvectors correctly <<<>>>\n"
                  " EXIT\n");
      if (r.fstop) throw DeckError{"the final eigenstates did not converge"};
    }
    // SPECTRUMTI (spectrumti.f:52-94): the initial states come back from the
    // file initial_spc.aux, written as E20.12 (12 significant digits)
    auto e20 = [](double x) {
      char b[40];
      std::snprintf(b, sizeof b, "%.11E", x);
      return std::strtod(b, nullptr);
    };
    std::printf(" \n Spectrum:\n =========\n");
    std::printf("     *E/a.u.*        *AMPT*           *FC*              *I->F*\n");
    for (int k = iil; k < iil + nis; ++k) {
      const double ei = e20(eval[k]);
      for (int j = r.ifl; j < r.ifl + r.nfs; ++j) {
        double w = 0.0;
        for (int i = 0; i < n; ++i) w += vecf[(size_t)j * n + i] * e20(eigvc[(size_t)k * n + i]);
        std::printf(" %12.7f    %12.7f    %12.7f          %2d ->%2d\n", evf[j] - ei, w, w * w,
                    k, j);
      }
    }
    eigvc.clear();
    return fd;
  }
  // FORMAT 1031 and the list-directed 'state started' line (espec.f:1083-1108)
  const int k = r.prpgstate - iil;
  const char* th = k == 1 ? "st" : k == 2 ? "nd" : k == 3 ? "rd" : "th";
  std::printf("\n%33sStarting %s%s state to be propagated...\n%12d %s state started.\n", "",
              k < 10 ? std::to_string(k).c_str() : "*", th, k, th);
  fd.psi.assign(eigvc.begin() + (size_t)r.prpgstate * n,
                eigvc.begin() + (size_t)(r.prpgstate + 1) * n);
  eigvc.erase(eigvc.begin(), eigvc.begin() + (size_t)iil * n);
  eigvc.resize((size_t)nis * n);
  return fd;
}

// espec.f:631-641, 818-830: the grid step in bohr; above 4e-2 the run stops
void check_step(const Run& r, const double* sh) {
  for (int a = 0; a < r.nd; ++a) {
    if (sh[a] > 4.0e-2) {
      std::printf(" <<<>>> Step bigger than%s  a.u. <<<>>>\n", list_real(4.0e-2).c_str());
      if (r.fstop) throw DeckError{"the grid step is above 4e-2 bohr"};
    } else if (sh[a] > 1.0e-2) {
      std::printf(" -> Warning step bigger than%s  a.u. !\n", list_real(1.0e-2).c_str());
    }
  }
}

// .ONLYSPEC (espec.f:1596-1626): the correlation function of an earlier run's
// output (GETCORR, getcorr.f: the 2^MF rows after its " Correlation
// Function:" line, DTF from the first two times and TF = last time + DTF),
// printed again with *PRTCRL, then HWHM and SPECTRUMTD
int only_spectrum(Run& r, const std::string& dir) {
  const std::string path = !r.fileaux.empty() && r.fileaux[0] == '/' ? r.fileaux : dir + r.fileaux;
  const int n2 = 1 << r.mf, mc = n2 / 2;
  msg1003("   Getting correlation function...");
  std::ifstream f(path);
  if (!f) {
    std::printf(" <<<>>> File %s cannot be open <<<>>>\n Please check and resubimit \n",
                r.fileaux.c_str());
    throw DeckError{"correlation file \"" + path + "\" cannot be opened"};
  }
  std::string line;
  bool found = false;
  while (std::getline(f, line))
    if (line.compare(0, 22, " Correlation Function:") == 0) {
      found = true;
      break;
    }
  if (!found) {
    std::printf(" <<<>>> Correlation function wasn`t found <<<>>>\n");
    throw DeckError{"no correlation function in " + path};
  }
  std::getline(f, line);
  std::getline(f, line);
  std::vector<double> t(n2), cu(n2), cv(n2);
  for (int i = 0; i < n2; ++i) {
    std::vector<double> x;
    if (!std::getline(f, line) || (x = numbers(line)).size() < 3) {
      std::printf(" <<<>>> Error reading correlation function <<<>>>\n");
      throw DeckError{"the correlation function in " + path + " has fewer than 2^MF rows"};
    }
    t[i] = x[0];
    cu[i] = x[1];
    cv[i] = x[2];
  }
  double dtf = t[1] - t[0];
  const double tf = t[n2 - 1] + dtf;
  std::printf(" Correlation function got.\n");
  if (starts(r.prtcrl, ".YES") || starts(r.prtcrl, ".PARTIAL"))
    std::printf("%s", correlation_table(mc, tf, cu, cv, dtf).c_str());
  double tff = tf;
  if (r.lhwhm) {
    double dde = r.de - r.e1i;
    msg1003("Appling the half-width at half-maximum...");
    std::fflush(stdout);
    hwhm_(&r.mf, &dtf, &tff, &r.chwhm, &dde, cu.data(), cv.data());
    std::printf(" Half-width at half-maximum applied.\n");
  }
  msg1003("   Processing spectrum...");
  std::fflush(stdout);
  double ade = r.ade;
  spectrumtd_(r.tpwind.c_str(), &r.mf, &dtf, &tff, &r.wp, &ade, cu.data(), cv.data(),
              r.tpwind.size());
  std::printf(" Spectrum done.\n \n The eSPec program finished successfully!\n");
  std::fflush(stdout);
  return ESPEC_OK;
}

int run_deck(const std::string& deck_path) {
  Run r = load_run(deck_path);
  const size_t slash = deck_path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string() : deck_path.substr(0, slash + 1);
  if (r.onlyspec()) return only_spectrum(r, dir);
  const std::string file = !r.potfile.empty() && r.potfile[0] == '/' ? r.potfile : dir + r.potfile;
  int n = 1;
  for (int a = 0; a < r.nd; ++a) n *= r.np[a];
  double sh[3] = {1, 1, 1}, shm[3] = {0, 0, 0}, sm[3] = {1, 1, 1};
  FileData fd;
  std::vector<double> eigvc;  // the computed states IIL..IIU (.CALC)
  if (r.calc() || r.pes()) {
    // espec.f:646-664: absorber bounds in angstrom unless the form is in bohr
    if (r.absorb && !starts(r.tpabsor, ".SMOOTHW_au") && !starts(r.tpabsor, ".SMRS_au") &&
        !starts(r.tpabsor, ".VOPTIC"))
      for (int a = 0; a < r.nd; ++a) {
        r.al[a] = r.al[a] / kA0A;
        r.ar[a] = r.ar[a] / kA0A;
      }
    for (int a = 0; a < r.nd; ++a) sh[a] = ((r.gxf[a] - r.gxi[a]) / (r.np[a] - 1.0)) / kA0A;
    check_step(r, sh);
    fd = initial_state(r, sh, shm, sm, eigvc);
    if (r.ti_form() || r.pes()) {  // no propagation (espec.f:881, 954, 1015-1080)
      std::printf(" \n The eSPec program finished successfully!\n");
      std::fflush(stdout);
      return ESPEC_OK;
    }
  } else {
    fd = read_file(file, n, r.nd, r.shiftp);
    for (int a = 0; a < r.nd; ++a) {
      sm[a] = kAmu * r.sm[a];  // espec.f:614
      sh[a] = (fd.xf[a] - fd.xi[a]) / (r.np[a] - 1.0);
      shm[a] = 1.0 / ((((24.0 * sm[a]) * r.smf[a]) * sh[a]) * sh[a]);  // espec.f:819
    }
    check_step(r, sh);
  }
  const int nc = c_stride(r);
  std::vector<double> vabc(n, 0.0);
  if (r.absorb)
    vabc = absorber_table(r.nd, r.np, r.tpabsor, r.al, r.ar, sh, fd.xi, fd.xf, r.voi);
  // propagation: the reference's LNZVC (its EIGVC) holds the computed states
  // in columns 1..NIS, the Lanczos basis in columns 1..MP and C(t) in MP+1,
  // MP+2 (espec.f:1357-1359)
  const int steps = (int)std::lround((r.tf - r.ti) / r.dt) + 4;
  const int mxdct = std::max(n, steps / nc + 4);
  const int mpr = r.mp + 1, mpi = r.mp + 2;
  const int ncol = std::max({r.mp + 2, r.nis, r.kp + r.npr + 1});
  std::vector<double> lnzvc((size_t)mxdct * ncol, 0.0);
  for (size_t j = 0; j < eigvc.size() / (n ? n : 1); ++j)
    std::copy(eigvc.begin() + j * n, eigvc.begin() + (j + 1) * n, lnzvc.begin() + j * mxdct);
  std::vector<double> u1 = fd.psi, v1 = fd.psi_im, u2(n, 0.0), v2(n, 0.0), tc(n, 0.0), wrk(n, 0.0);
  v1.resize(n, 0.0);
  const int absorb = r.absorb ? 1 : 0, lmt = 10, change = r.change ? 1 : 0;
  double abstol = 1e-6;
  std::vector<int> iwork(64, 0);
  const double xi0 = 0.0;
  int info = 0, mp = r.mp;
  const char* pr = r.prtcrl.c_str();
  const char* dm = r.dim.c_str();
  const char* ta = r.tpabsor.empty() ? ".NONE" : r.tpabsor.c_str();
  msg1003("Propagating eigenvector...");
  // espec.f:1361-1498
  const char* using_msg = starts(r.tppropg, ".PFSPO")   ? "Using SPO procedure with FFT."
                          : starts(r.tppropg, ".PFSOD") ? "Using SOD procedure with FFT."
                          : starts(r.tppropg, ".PSIL")  ? "Using SIL procedure."
                          : starts(r.tppropg, ".PSOD")  ? "Using SOD procedure."
                          : starts(r.tppropg, ".PPSOD")
                              ? "Using time dependent SOD procedure with pulse and printing facilities."
                          : starts(r.tppropg, ".PPSIL") || starts(r.tppropg, ".PPLNZ")
                              ? "Using time dependent SIL procedure with pulse and printing facilities."
                              : nullptr;
  if (using_msg) std::printf(" %s\n", using_msg);
  std::fflush(stdout);
  if (starts(r.tppropg, ".PFSPO")) {
    pspofft_(&absorb, dm, pr, ta, &info, &nc, &mp, &mpi, &mpr, &mxdct, &n, &r.dt, &r.ti, &r.tf,
             &r.tol, r.np, shm, sh, sm, u1.data(), v1.data(), &xi0, &xi0, tc.data(),
             fd.vpot.data(), vabc.data(), lnzvc.data(), wrk.data(), wrk.data(), &xi0,
             std::strlen(dm), std::strlen(pr), std::strlen(ta));
  } else if (starts(r.tppropg, ".PFSOD")) {
    psodfft_(&absorb, dm, pr, ta, &info, &nc, &mp, &mpi, &mpr, &mxdct, &n, &r.dt, &r.ti, &r.tf,
             &r.tol, r.np, shm, sh, sm, u1.data(), u2.data(), v1.data(), v2.data(), &xi0, &xi0,
             tc.data(), fd.vpot.data(), vabc.data(), wrk.data(), wrk.data(), &xi0, lnzvc.data(),
             std::strlen(dm), std::strlen(pr), std::strlen(ta));
  } else if (starts(r.tppropg, ".PSIL")) {
    plnz_(&absorb, &change, dm, pr, ta, &info, &nc, &lmt, &mp, &mpi, &mpr, &mxdct, &n, &abstol,
          &r.dt, &r.ti, &r.tf, &r.tol, r.np, iwork.data(), shm, fd.vpot.data(), vabc.data(),
          u1.data(), v1.data(), &xi0, &xi0, wrk.data(), wrk.data(), wrk.data(), wrk.data(), &xi0,
          lnzvc.data(), std::strlen(dm), std::strlen(pr), std::strlen(ta));
  } else if (starts(r.tppropg, ".PSOD")) {
    psod_(&absorb, dm, pr, ta, &info, &nc, &mp, &mpi, &mpr, &mxdct, &n, &r.dt, &r.ti, &r.tf,
          &r.tol, r.np, shm, u1.data(), u2.data(), v1.data(), v2.data(), &xi0, &xi0,
          fd.vpot.data(), vabc.data(), wrk.data(), &xi0, lnzvc.data(), std::strlen(dm),
          std::strlen(pr), std::strlen(ta));
  } else if (starts(r.tppropg, ".PPSOD") || starts(r.tppropg, ".PPSIL") ||
             starts(r.tppropg, ".PPLNZ")) {
    // DIPLMMT (dipl.f:61-95): R = XI(1) + (I - 1) SH(1) for every I of the
    // grid, or the values of a file read as RDPTE reads (which sets XI, XF
    // again from its coordinates)
    std::vector<double> dmv(n, 0.0);
    if (starts(r.tpdipl, ".READ")) {
      const std::string dmf = !r.dmfile.empty() && r.dmfile[0] == '/' ? r.dmfile : dir + r.dmfile;
      std::ifstream f(dmf);
      if (!f) throw DeckError{"dipole file \"" + dmf + "\" cannot be opened"};
      read_block(f, dmf, n, r.nd, dmv, fd.xi, fd.xf);
    }
    for (int i = 0; i < n && !starts(r.tpdipl, ".READ"); ++i) {
      const double rab = fd.xi[0] + i * sh[0];
      if (starts(r.tpdipl, ".CONST")) {
        dmv[i] = r.cstdm[0] / rab;
      } else if (starts(r.tpdipl, ".EXP+")) {  // normalised at the final surface's Re
        const double c = r.cstdm[1], re = r.cstf[0];
        dmv[i] = r.cstdm[0] * (std::exp(-c * rab) - std::exp(-3.0 * c * rab)) /
                 (std::exp(-c * re) - std::exp(-3.0 * c * re));
      } else if (starts(r.tpdipl, ".EXP")) {
        dmv[i] = r.cstdm[0] * rab * std::exp(-r.cstdm[1] * rab);
      }
    }
    const int off = 0, nshot = 10, nispg = r.prpgstate + 1;  // espec.f:240
    const char* ef = r.efc.c_str();
    if (!starts(r.tppropg, ".PPSOD")) {  // espec.f:1513-1518
      pplnz_(&absorb, &change, &off, &off, &off, dm, ef, pr, ta, &info, &nc, &lmt, &mp, &mpi,
             &mpr, &mxdct, &n, &nshot, &r.kl, &r.npr, &r.kp, &abstol, &r.dt, &r.ti, &r.tf, &r.tol,
             &r.e0, &r.t0, &r.td, &r.tp, &r.omg, &r.sni, r.np, r.np, iwork.data(), sh, shm,
             fd.vpot.data(), vabc.data(), u1.data(), v1.data(), fd.xi, fd.xf, fd.xi, dmv.data(),
             wrk.data(), wrk.data(), wrk.data(), wrk.data(), &xi0, lnzvc.data(), std::strlen(dm),
             std::strlen(ef), std::strlen(pr), std::strlen(ta));
    } else {
      ppsod_(&absorb, &off, &off, &off, dm, ef, pr, ta, &info, &nc, &mp, &mpi, &mpr, &mxdct, &n,
             &nshot, &r.npr, &r.kp, &nispg, &r.e0, &r.t0, &r.td, &r.tp, &r.omg, &r.sni, &r.kl,
             &r.dt, &r.ti, &r.tf, &r.tol, r.np, r.np, sh, shm, u1.data(), u2.data(), v1.data(),
             v2.data(), fd.xi, fd.xi, fd.xf, dmv.data(), fd.vpot.data(), vabc.data(), wrk.data(),
             &xi0, lnzvc.data(), &off, &off, &xi0, &off, std::strlen(dm), std::strlen(ef),
             std::strlen(pr), std::strlen(ta));
    }
  } else {
    throw DeckError{"propagator " + r.tppropg + " is not covered (.PFSPO, .PFSOD, .PSIL, .PSOD, "
                    ".PPSOD, .PPSIL, .PPLNZ)"};
  }
  if (info == 2) throw DeckError{"the GPU propagation failed (INFO = 2)"};
  if (info != 0) {
    std::printf(" <<<>>> Propagation operator error <<<>>>\n INFO =%12d\n", info);
    if (r.fstop) throw DeckError{"propagation operator error (INFO = 1)"};
  }
  std::printf(" Eigenvector propagated.\n");
  if (starts(r.tpclc, ".PROPAGATION") || r.collision()) {  // espec.f:1541-1542
    std::printf(" \n The eSPec program finished successfully!\n");
    return ESPEC_OK;
  }
  // total correlation (espec.f:1545-1576): C(-t) = C(t)*, 2^MF samples
  msg1003("Calculating total correlation function...");
  const int mc = (int)(std::pow(2.0, r.mf) / 2.0);
  const double dtf = r.tf / mc;
  std::vector<double> cu, cv;
  total_correlation(mc, lnzvc.data() + (size_t)(mpr - 1) * mxdct,
                    lnzvc.data() + (size_t)(mpi - 1) * mxdct, cu, cv);
  std::printf(" Total correlation function calculated.\n%s",
              correlation_table(mc, r.tf, cu, cv).c_str());
  if (starts(r.tpclc, ".CORRELATION")) {
    std::printf(" \n The eSPec program finished successfully!\n");
    return ESPEC_OK;
  }
  if (r.lhwhm) {
    double dde = r.de - r.e1i;
    msg1003("Appling the half-width at half-maximum...");
    std::fflush(stdout);
    hwhm_(&r.mf, &dtf, &r.tf, &r.chwhm, &dde, cu.data(), cv.data());
    std::printf(" Half-width at half-maximum applied.\n");
  }
  msg1003("   Processing spectrum...");
  std::fflush(stdout);
  double ade = r.ade;
  spectrumtd_(r.tpwind.c_str(), &r.mf, &dtf, &r.tf, &r.wp, &ade, cu.data(), cv.data(),
              r.tpwind.size());
  std::printf(" Spectrum done.\n \n The eSPec program finished successfully!\n");
  std::fflush(stdout);
  return ESPEC_OK;
}

// One deck, K .FILE inputs (initial state and potential each), 1D .PFSPO or
// .PFSOD: one batched plan over all K packets, one batched spectrum launch,
// per packet the total correlation and spectrum blocks written to
// <prefix><k>.crl and <prefix><k>.spc (k from 1).
int run_scan(const std::string& deck_path, int njobs, const char* const* files,
             const std::string& prefix) {
  Run r = load_run(deck_path);
  if (r.nd != 1) throw DeckError{"scans run 1D decks (the batched plans are 1D)"};
  if (r.calc()) throw DeckError{"scans read their states from .FILE inputs (.GETR)"};
  const bool spo = starts(r.tppropg, ".PFSPO");
  if (!spo && !starts(r.tppropg, ".PFSOD"))
    throw DeckError{"scans run .PFSPO or .PFSOD (the batched plans)"};
  if (!starts(r.tpclc, ".SPECTRUM")) throw DeckError{"scans produce spectra: *TPCALC .SPECTRUM .TD"};
  if (njobs < 1 || !files) throw DeckError{"no input files"};
  const size_t slash = deck_path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string() : deck_path.substr(0, slash + 1);
  const int n = r.np[0];
  const double sm = kAmu * r.sm[0];
  std::vector<double> vpot((size_t)njobs * n), psi((size_t)njobs * n), vabc;
  std::vector<double> sh(njobs), sms(njobs, sm);
  std::vector<int> npts(njobs, n);
  if (r.absorb) vabc.resize((size_t)njobs * n);
  for (int k = 0; k < njobs; ++k) {
    const std::string f = files[k][0] == '/' ? std::string(files[k]) : dir + files[k];
    FileData fd = read_file(f, n, 1, r.shiftp);
    sh[k] = (fd.xf[0] - fd.xi[0]) / (n - 1.0);
    std::copy(fd.psi.begin(), fd.psi.end(), psi.begin() + (size_t)k * n);
    std::copy(fd.vpot.begin(), fd.vpot.end(), vpot.begin() + (size_t)k * n);
    if (r.absorb) {
      const double shk = sh[k];
      const std::vector<double> t =
          absorber_table(1, r.np, r.tpabsor, r.al, r.ar, &shk, fd.xi, fd.xf, r.voi);
      std::copy(t.begin(), t.end(), vabc.begin() + (size_t)k * n);
    }
  }
  const int nc = c_stride(r);
  const int ab = !r.absorb ? ESPEC_ABS_NONE
                           : (starts(r.tpabsor, ".VOPTIC") ? ESPEC_ABS_VOPTIC : ESPEC_ABS_SMOOTHW);
  const int quirks = spo ? ESPEC_Q_SPO_INPLACE : ESPEC_Q_SOD_SMOOTHW;
  // step counts of the drop-ins (pspofft.f:110; psodfft.f:120-154)
  const int nsteps = spo ? do_count_real(r.ti + r.dt, r.tf + r.dt, r.dt)
                         : 1 + do_count_real(r.ti + 2 * r.dt, r.tf + r.dt, r.dt);
  const int mc = (int)(std::pow(2.0, r.mf) / 2.0);
  if ((long)(mc - 1) * nc > nsteps) throw DeckError{"fewer C(t) samples than 2^(MF-1)"};
  espec_spo_plan* plan = nullptr;
  struct Guard {
    espec_spo_plan*& p;
    ~Guard() { espec_spo_destroy(p); }
  } guard{plan};
  std::vector<double> cre((size_t)njobs * (nsteps + 1)), cim(cre.size());
  if (espec_prop_create(&plan, njobs, npts.data(), sh.data(), sms.data(), r.dt,
                        spo ? ESPEC_SPO : ESPEC_SOD, ESPEC_FP64, ab, quirks) ||
      espec_spo_load(plan, vpot.data(), r.absorb ? vabc.data() : nullptr, psi.data(), nullptr,
                     ESPEC_MEM_HOST, nullptr) ||
      espec_spo_run(plan, nsteps, nullptr) ||
      espec_spo_results(plan, cre.data(), cim.data(), nullptr, nullptr, ESPEC_MEM_HOST, nullptr))
    throw DeckError{std::string("batched propagation: ") + espec_last_error()};
  // every NC-th sample (the LNZVC rows of the drop-ins), packed per packet
  std::vector<double> cpk((size_t)njobs * mc * 2);
  for (int k = 0; k < njobs; ++k)
    for (int s = 0; s < mc; ++s) {
      const size_t src = (size_t)k * (nsteps + 1) + (size_t)s * nc;
      cpk[((size_t)k * mc + s) * 2] = cre[src];
      cpk[((size_t)k * mc + s) * 2 + 1] = cim[src];
    }
  const size_t N = (size_t)1 << r.mf;
  const double dtf = r.tf / mc;
  int window = -1;
  if (starts(r.tpwind, ".SG")) window = 1;
  else if (starts(r.tpwind, ".NONE") || starts(r.tpwind, ".NULL")) window = 0;
  if (window < 0) throw DeckError{"*WINDOWING " + r.tpwind + " is not defined (spectrumtd.f)"};
  void *d_in = nullptr, *d_spec = nullptr, *d_work = nullptr;
  struct Free {
    void** p[3];
    ~Free() {
      for (void** q : p)
        if (*q) cudaFree(*q);
    }
  } fr{{&d_in, &d_spec, &d_work}};
  std::vector<double> spec((size_t)njobs * N * 2);
  if (cudaMalloc(&d_in, cpk.size() * 8) != cudaSuccess ||
      cudaMalloc(&d_spec, spec.size() * 8) != cudaSuccess ||
      cudaMalloc(&d_work, espec_spectrum_work_bytes(njobs, r.mf)) != cudaSuccess ||
      cudaMemcpy(d_in, cpk.data(), cpk.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    throw DeckError{"device buffers for the spectra"};
  if (espec_spectrum_dev(njobs, r.mf, d_in, mc, 1, dtf, r.tf, r.lhwhm ? r.chwhm : -1.0,
                         r.de - r.e1i, window, r.wp, ESPEC_Q_FFTNT_SP, d_spec, d_work, nullptr) ||
      cudaMemcpy(spec.data(), d_spec, spec.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    throw DeckError{std::string("batched spectrum: ") + espec_last_error()};
  const double ade = r.ade < 0.0 ? 0.0 : r.ade;  // spectrumtd.f: DE < 0 is set to 0
  std::vector<double> cr(mc), ci(mc), cu, cv, u(N), v(N);
  for (int k = 0; k < njobs; ++k) {
    for (int s = 0; s < mc; ++s) {
      cr[s] = cpk[((size_t)k * mc + s) * 2];
      ci[s] = cpk[((size_t)k * mc + s) * 2 + 1];
    }
    total_correlation(mc, cr.data(), ci.data(), cu, cv);
    for (size_t i = 0; i < N; ++i) {
      u[i] = spec[((size_t)k * N + i) * 2];
      v[i] = spec[((size_t)k * N + i) * 2 + 1];
    }
    const std::string base = prefix + std::to_string(k + 1);
    std::ofstream fc(base + ".crl"), fs(base + ".spc");
    if (!fc || !fs) throw DeckError{"cannot write " + base + ".crl / .spc"};
    fc << correlation_table(mc, r.tf, cu, cv);
    fs << espec::spectrum_table(r.mf, dtf, ade, u.data(), v.data());
  }
  return ESPEC_OK;
}

}  // namespace

extern "C" int espec_run_scan(const char* deck_path, int njobs, const char* const* data_files,
                              const char* out_prefix) {
  if (!deck_path || !out_prefix) return espec::set_error(ESPEC_EINVAL, "null argument");
  try {
    return run_scan(deck_path, njobs, data_files, out_prefix);
  } catch (const DeckError& e) {
    std::fflush(stdout);
    std::fprintf(stderr, "espec_gpu scan: %s\n", e.what.c_str());
    return espec::set_error(ESPEC_EINVAL, e.what.c_str());
  }
}

extern "C" int espec_run_deck(const char* deck_path) {
  if (!deck_path) return espec::set_error(ESPEC_EINVAL, "null deck path");
  try {
    return run_deck(deck_path);
  } catch (const DeckError& e) {
    std::fflush(stdout);
    std::fprintf(stderr, "espec_gpu deck: %s\n", e.what.c_str());
    return espec::set_error(ESPEC_EINVAL, e.what.c_str());
  }
}
