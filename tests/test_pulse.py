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


def test_pplnz_call_times():
    """PPLNZ's DO T = TI+DT, TF+DT/2, DT (pplnz.f:200): the real DO loop's trip
    count INT((TF + DT/2 - (TI + DT) + DT)/DT), T accumulating DT."""
    par = (1e12, 0.5, 2.0, 0.7, 0.3)
    ti, dt, tf = 0.05, 0.01, 0.4
    ef = GR.pplnz_field(N.PULSE_GAUS, par, ti, tf, dt)
    nt = int((tf + dt / 2 - (ti + dt) + dt) / dt)
    assert len(ef) == nt + 1
    t = ti + dt
    for s in range(1, nt + 1):
        assert ef[s] == GR.pulse_field(N.PULSE_GAUS, par, t)
        t = t + dt


@pytest.mark.parametrize("ndim", [1, 2])
def test_oracle_tables_agree_with_propagations(oracle, ndim):
    """The oracle's PPSOD and PPLNZ with their tables (orc_ppsod_table,
    orc_pplnz_table) store the same C(t) and leave the same psi as the plain
    propagations (orc_ppsod, orc_pplnz) with .YES printing and LC = 1."""
    np_ = [64] if ndim == 1 else [24, 20]
    n = int(np.prod(np_))
    axes = [np.linspace(-1.0, 1.0, k) * (0.6 + 0.2 * a) for a, k in enumerate(np_)]
    grids = np.meshgrid(*axes, indexing="ij")
    v = sum(0.5 * g ** 2 for g in grids).ravel(order="F")
    psi = np.exp(-sum((g - 0.1) ** 2 / 0.08 for g in grids)) * np.exp(1j * 2.0 * grids[0])
    psi = (psi / np.sqrt(np.sum(np.abs(psi) ** 2))).ravel(order="F")
    sh = [ax[1] - ax[0] for ax in axes]
    sm = [1000.0] * ndim
    dm = (0.8 * grids[0]).ravel(order="F")
    par = (6e7, 0.08, 2.5, 0.12, 0.3)
    dt = 0.0005 * N.SHFS
    p = oracle.make_prop(np_, dt, 0.0, 0.02, sh, sm, lc=1, prtcrl=oracle.PRT_YES, mp=8,
                         lmtreort=16, change=0, quirks=oracle.Q_SIL_INPLACE)
    a = oracle.ppsod(p, v, dm, N.PULSE_GAUS, par, psi.real, psi.imag)
    b = oracle.ppsod_table(p, v, dm, N.PULSE_GAUS, par, np.zeros((0, n)), psi.real, psi.imag)
    assert np.array_equal(a["c"], b["c"])
    assert np.array_equal(a["u"], b["u"]) and np.array_equal(a["v_prev"], b["v_prev"])
    assert b["rows"].shape[0] == len(b["c"])  # .YES: a row per stored sample
    c = oracle.pplnz(p, v, dm, N.PULSE_GAUS, par, psi.real, psi.imag)
    d = oracle.pplnz_table(p, v, dm, N.PULSE_GAUS, par, 1, np.zeros((1, n)), psi.real, psi.imag)
    assert np.array_equal(c["c"], d["c"])
    assert np.array_equal(c["u"], d["u"]) and np.array_equal(c["v"], d["v"])
    np.testing.assert_allclose(d["rows"][:, 5], np.abs(d["c"]) ** 2, rtol=1e-14)
