// pulse.cpp -- the laser field of eSPec's pulse-driven propagators: EF
// (ef.f:20-60) for the pulse shapes, and the field of every step of a PPSOD
// run (ppsod.f:252-260, 378-386) or a PPLNZ run (pplnz.f:139-141), the tables
// espec_grid_set_pulse takes.
#include <cmath>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace {
// ef.f:40-43
const double kFat = 2.1132e-9;
const double kFate = 2.29371276e17 * 3.335664e-28;  // V/cm -> a.u./D
const double kFatt = 1.5192676;
const double kPi = 3.14159265358979323846;
}  // namespace

extern "C" double espec_pulse_field(int shape, const double* par, double t) {
  if (!par) return 0.0;
  const double e0 = par[0], tp = par[1], omg = par[2], t0 = par[3], sni = par[4];
  switch (shape) {
    case ESPEC_PULSE_GAUS: {  // ef.f:45-48
      const double ef = e0 * std::exp(-4.0 * 0.693147181 * (t - t0) * (t - t0) / (tp * tp)) *
                        std::cos(omg * t * kFatt + sni);
      return ef * kFate;
    }
    case ESPEC_PULSE_GGAUS: {  // ef.f:49-53; 0.693147181 is a REAL (single) literal there
      const int kl = (int)par[5];
      const double a1 = 1.0 / (2.0 * kl);
      const double tpa = tp / std::pow((double)0.693147181f, a1);
      return kFat * std::sqrt(e0 * std::exp(-std::pow((t - t0) / tpa, 2.0 * kl))) *
             std::cos(omg * t * kFatt + sni);
    }
    case ESPEC_PULSE_SIN2: {  // ef.f:54-57 (par[3] is the delay TD)
      const double ef = e0 * std::cos(kPi * (t - t0) / tp) * std::cos(kPi * (t - t0) / tp) *
                        std::cos(omg * (t - t0) * kFatt + sni);
      return ef * kFate;
    }
    default:
      return 0.0;
  }
}

extern "C" long espec_ppsod_field(int shape, const double* par, double ti, double tf, double dt,
                                  double* ef, long cap) {
  if (!ef || cap < 2 || dt <= 0.0) return espec::set_error(ESPEC_EINVAL, "bad field table");
  // start-up at (T + DT)/2 and T + DT with T = TI (ppsod.f:252-258)
  ef[0] = espec_pulse_field(shape, par, (ti + dt) / 2.0);
  ef[1] = espec_pulse_field(shape, par, ti + dt);
  // NF = NINT((TF + DT/2 - T)/DT) steps from T = TI + DT, T accumulating DT
  double t = ti + dt;
  const long nf = std::lround((tf + dt / 2.0 - t) / dt);
  if (nf + 2 > cap) return espec::set_error(ESPEC_EINVAL, "field table too short");
  for (long k = 1; k <= nf; ++k) {
    t = t + dt;
    ef[1 + k] = espec_pulse_field(shape, par, t);
  }
  return nf + 2;
}

extern "C" long espec_pplnz_field(int shape, const double* par, double ti, double tf, double dt,
                                  double* ef, long cap) {
  if (!ef || cap < 1 || dt <= 0.0) return espec::set_error(ESPEC_EINVAL, "bad field table");
  // DO T = TI+DT, TF+DT/2, DT (pplnz.f:139): CHPOT(T) before each step
  const double x = (tf + dt / 2.0 - (ti + dt) + dt) / dt;
  const long nt = x > 0.0 ? (long)x : 0;
  if (nt + 1 > cap) return espec::set_error(ESPEC_EINVAL, "field table too short");
  ef[0] = espec_pulse_field(shape, par, ti);
  double t = ti + dt;
  for (long s = 1; s <= nt; ++s) {
    ef[s] = espec_pulse_field(shape, par, t);
    t = t + dt;
  }
  return nt + 1;
}
