"""GPU parity of the pulse-driven second-order-differences propagation
(PPSOD's time loop, ppsod.f with chpot.f and ef.f) against the oracle's
restatement, FP64: |dC(t)|, |dpsi(TF)|, |dpsi(TF - dt)| <= 1e-10 with the
potential V - DM EF(t) changing every step."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT
from espec_b200 import grid as GR

import golden_cases as G
from test_gpu_psod import packet

pytestmark = pytest.mark.gpu

PULSES = {"gaus": (NAT.PULSE_GAUS, (6e7, 0.08, 2.5, 0.12, 0.3)),
          "ggaus": (NAT.PULSE_GGAUS, (3e11, 0.08, 2.5, 0.12, 0.3, 2)),
          "sin2": (NAT.PULSE_SIN2, (6e7, 0.2, 3.0, 0.05, 0.0))}


@pytest.mark.parametrize("np_,pulse,absorb", [
    ([301], "gaus", 0), ([256], "ggaus", 1), ([300], "sin2", 2), ([40, 36], "gaus", 0),
    ([48, 33], "sin2", 1), ([10, 12, 9], "gaus", 0)])
def test_ppsod_matches_oracle(oracle, np_, pulse, absorb):
    v, psi, sh, grids = packet(np_, sum(np_) + 7)
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dm = (0.8 * grids[0] + 0.3 * grids[0] ** 2).ravel(order="F")  # dipole function
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.05 * np.clip(grids[0] - 0.3, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F")
    shape, par = PULSES[pulse]
    dt, ti, tf = 0.002 * NAT.SHFS, 0.0, 0.25
    p = oracle.make_prop(np_, dt, ti, tf, sh, sm, lc=1, absorb=absorb, shm=shm)
    ref = oracle.ppsod(p, v, dm, shape, par, np.real(psi), np.imag(psi), vabc=vabc)
    ef = GR.ppsod_field(shape, par, ti, tf, dt)
    assert np.max(np.abs(ef)) > 1e-4  # the pulse moves the potential
    g = E.PsodGrid(np_, shm, dt, absorb=absorb)
    g.load(v, psi, vabc=vabc)
    g.set_pulse(dm, ef)
    g.run(len(ef) - 1)
    c, out = g.results()
    prev = g.previous()
    g.close()
    assert len(c) == ref["nc"]
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10
    # the field mattered: the same run without it differs
    ref0 = oracle.ppsod(p, v, dm, NAT.PULSE_NONE, par, np.real(psi), np.imag(psi), vabc=vabc)
    assert np.max(np.abs(ref0["c"] - ref["c"])) > 1e-6


def test_ppsod_continue_and_field_energies(oracle):
    np_ = [64, 48]
    v, psi, sh, grids = packet(np_, 5)
    sm = [918.0, 1500.0]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dm = (0.5 * grids[0]).ravel(order="F")
    shape, par = PULSES["gaus"]
    dt = 0.002 * NAT.SHFS
    ef = GR.ppsod_field(shape, par, 0.0, 0.2, dt)
    one = E.PsodGrid(np_, shm, dt)
    one.load(v, psi)
    one.set_pulse(dm, ef)
    one.run(len(ef) - 1)
    c1, p1 = one.results()
    seg = E.PsodGrid(np_, shm, dt)
    seg.load(v, psi)
    seg.set_pulse(dm, ef)
    seg.run(40)
    ca, _ = seg.results()
    seg.advance(len(ef) - 1 - 40)
    cb, p2 = seg.results()
    assert np.max(np.abs(np.concatenate([ca, cb[1:]]) - c1)) <= 1e-12
    assert np.max(np.abs(p2 - p1)) <= 1e-12
    with pytest.raises(NAT.EspecError):
        seg.advance(5)  # past the end of the field table
    e, nr = seg.energies_at(ef[-1])
    veff = v - dm * ef[-1]
    ref_e = oracle.eigenerg(np_, shm, veff, p2.real) + oracle.eigenerg(np_, shm, veff, p2.imag)
    assert abs(e - ref_e) <= 1e-12 * abs(ref_e)
    e0, _ = seg.energies_at(0.0)
    ref_e0 = oracle.eigenerg(np_, shm, v, p2.real) + oracle.eigenerg(np_, shm, v, p2.imag)
    assert abs(e0 - ref_e0) <= 1e-12 * abs(ref_e0)
    one.close()
    seg.close()


@pytest.mark.parametrize("np_,pulse,mask,mp", [([301], "gaus", False, 10), ([256], "sin2", True, 12),
                                              ([40, 36], "ggaus", False, 8),
                                              ([10, 12, 9], "gaus", True, 6)])
def test_pplnz_matches_oracle(oracle, np_, pulse, mask, mp):
    """PPLNZ's time loop (pplnz.f:139-141): SIL steps with V - DM EF(T) at the
    time each step lands at."""
    v, psi, sh, grids = packet(np_, sum(np_) + mp)
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dm = (0.8 * grids[0] + 0.3 * grids[0] ** 2).ravel(order="F")
    vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F") if mask else None
    absorb = NAT.ABS_SMOOTHW if mask else NAT.ABS_NONE
    shape, par = PULSES[pulse]
    dt, ti, tf = 0.02 * NAT.SHFS, 0.0, 0.2
    p = oracle.make_prop(np_, dt, ti, tf, sh, sm, lc=1, absorb=absorb, mp=mp, lmtreort=16,
                         change=0, shm=shm)
    ref = oracle.pplnz(p, v, dm, shape, par, np.real(psi), np.imag(psi), vabc=vabc)
    ef = GR.pplnz_field(shape, par, ti, tf, dt)
    g = E.SilGrid(np_, shm, dt, mp, absorb=absorb)
    g.load(v, psi, vabc=vabc)
    g.set_pulse(dm, ef)
    g.run(len(ef) - 1)
    c, out = g.results()
    assert len(c) == ref["nc"]
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    e, _ = g.energies_at(ef[-1])
    veff = v - dm * ef[-1]
    ref_e = oracle.eigenerg(np_, shm, veff, out.real) + oracle.eigenerg(np_, shm, veff, out.imag)
    assert abs(e - ref_e) <= 1e-12 * abs(ref_e)
    g.close()
    ref0 = oracle.pplnz(p, v, dm, NAT.PULSE_NONE, par, np.real(psi), np.imag(psi), vabc=vabc)
    assert np.max(np.abs(ref0["c"] - ref["c"])) > 1e-6
