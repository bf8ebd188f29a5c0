"""Laser pulses of the pulse-driven propagators (ef.f, chpot.f, ppsod.f): the
library's field (espec_pulse_field, espec_ppsod_field) against the oracle's
restatement and closed-form values, on the CPU."""
import numpy as np
import pytest

from espec_b200 import _native as N
from espec_b200 import grid as GR

FATE = 2.29371276e17 * 3.335664e-28
FATT = 1.5192676


@pytest.mark.parametrize("shape,par", [
    (N.PULSE_GAUS, (1e12, 0.5, 2.0, 0.7, 0.3)),
    (N.PULSE_GGAUS, (1e12, 0.5, 2.0, 0.7, 0.3, 2)),
    (N.PULSE_SIN2, (1e12, 0.5, 2.0, 0.1, 0.3)),
    (N.PULSE_NONE, (1e12, 0.5, 2.0, 0.1, 0.3))])
def test_field_matches_oracle(oracle, shape, par):
    for t in np.linspace(-0.5, 2.0, 37):
        assert GR.pulse_field(shape, par, t) == pytest.approx(oracle.ef(shape, par, t),
                                                               rel=1e-14, abs=1e-30)


def test_field_closed_forms():
    # .GAUS at its peak: E0 cos(OMG T0 FATT + SNI) in a.u.
    e0, tp, omg, t0, sni = 1e12, 0.5, 2.0, 0.7, 0.3
    want = e0 * np.cos(omg * t0 * FATT + sni) * FATE
    assert GR.pulse_field(N.PULSE_GAUS, (e0, tp, omg, t0, sni), t0) == pytest.approx(want, 1e-14)
    # half maximum of the envelope at T0 +- TP/2
    r = GR.pulse_field(N.PULSE_GAUS, (e0, tp, 0.0, t0, 0.0), t0 + tp / 2) / (e0 * FATE)
    assert r == pytest.approx(0.5, abs=1e-9)
    # .SIN2 vanishes at TD +- TP/2
    assert abs(GR.pulse_field(N.PULSE_SIN2, (e0, tp, omg, 0.1, sni), 0.1 + tp / 2)) < 1e-20


def test_ppsod_call_times():
    par = (1e12, 0.5, 2.0, 0.7, 0.3)
    ti, dt, tf = 0.05, 0.01, 0.4
    ef = GR.ppsod_field(N.PULSE_GAUS, par, ti, tf, dt)
    nf = int(np.floor((tf + dt / 2 - (ti + dt)) / dt + 0.5))  # Fortran NINT: ties away from 0
    assert len(ef) == nf + 2
    assert ef[0] == GR.pulse_field(N.PULSE_GAUS, par, (ti + dt) / 2)  # (T + DT)/2, T = TI
    assert ef[1] == GR.pulse_field(N.PULSE_GAUS, par, ti + dt)
    t = ti + dt
    for k in range(1, nf + 1):
        t = t + dt
        assert ef[1 + k] == GR.pulse_field(N.PULSE_GAUS, par, t)
