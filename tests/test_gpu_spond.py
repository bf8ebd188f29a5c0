"""GPU parity of the 2D/3D split-operator propagator (PSPOFFT/PSPOFFTAUX on
N-D grids) against the oracle's restatement: FP64 |dC(t)|, |dpsi| <= 1e-10,
the reference's 2D kinetic-table and in-place defects included; the mixed
form against the FP64 form."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT

import golden_cases as G

pytestmark = pytest.mark.gpu


def oracle_spo(oracle, np_, sh, sm, dt, nsteps, v, psi, absorb=0, vabc=None, quirks=0):
    p = oracle.make_prop(np_, dt, 0.0, nsteps * dt, sh, sm, lc=1, absorb=absorb, quirks=quirks)
    nst = oracle.do_count(dt, nsteps * dt + dt, dt)
    return oracle.pspofft(p, v, np.real(psi).copy(), np.imag(psi).copy(), vabc=vabc), nst


def gpu_spo(np_, sh, sm, dt, v, psi, nsteps, precision="fp64", absorb=0, vabc=None, quirks=0):
    g = E.SpoGrid(np_, sh, sm, dt, precision=precision, absorb=absorb, quirks=quirks)
    g.load(v, psi, vabc=vabc)
    g.run(nsteps)
    c, out = g.results()
    g.close()
    return c, out


def packet(np_, seed):
    rng = np.random.default_rng(seed)
    axes = [np.linspace(0.6, 3.6, n) for n in np_]
    grids = np.meshgrid(*axes, indexing="ij")
    re = [1.4, 1.8, 2.0]
    v = sum((0.17 - 0.03 * a) * (1 - np.exp(-(1.0 + 0.2 * a) * (g - re[a]))) ** 2
            for a, g in enumerate(grids)) + 0.01 * (grids[0] - 1.4) * (grids[1] - 1.8)
    c0 = rng.uniform(1.6, 2.0, len(np_))
    psi = np.exp(-sum((g - c) ** 2 / (2 * 0.15 ** 2) for g, c in zip(grids, c0)))
    psi = psi * np.exp(1j * 2.0 * grids[0])
    psi = psi / np.sqrt(np.sum(np.abs(psi) ** 2))
    sh = [ax[1] - ax[0] for ax in axes]
    sm = [918.0, 1500.0, 1836.0][:len(np_)]
    return v.ravel(order="F"), psi.ravel(order="F"), sh, sm, grids


def test_golden_2d_spo_with_reference_defects(oracle):
    case = G.setup_case("morse2d_spo")
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_NONE)
    nsteps = ref["nc"] - 1
    c, psi = gpu_spo(case["np"], case["sh"], case["sm"], case["dt"], case["vpot"], case["psi"],
                     nsteps, quirks=NAT.Q_SPO_INPLACE | NAT.Q_DIGT_ND)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(psi - (ref["u"] + 1j * ref["v"]))) <= 1e-10


@pytest.mark.parametrize("np_,absorb", [([64, 128], 0), ([128, 32], 1), ([256, 64], 2),
                                        ([32, 64, 32], 0), ([64, 32, 32], 1)])
def test_nd_grids_match_oracle(oracle, np_, absorb):
    v, psi, sh, sm, grids = packet(np_, sum(np_))
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.02 * np.clip(grids[0] - 3.2, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 3.3, 0.97, 1.0).ravel(order="F")
    dt = 0.02 * NAT.SHFS
    ref, nst = oracle_spo(oracle, np_, sh, sm, dt, 60, v, psi, absorb=absorb, vabc=vabc)
    c, out = gpu_spo(np_, sh, sm, dt, v, psi, nst, absorb=absorb, vabc=vabc)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10


@pytest.mark.parametrize("np_", [[128, 128], [64, 64, 64]])
def test_mixed_form_against_fp64(np_):
    v, psi, sh, sm, _ = packet(np_, 5)
    dt = 0.1 * NAT.SHFS
    c64, p64 = gpu_spo(np_, sh, sm, dt, v, psi, 400)
    c32, p32 = gpu_spo(np_, sh, sm, dt, v, psi, 400, precision="mixed")
    # 400 steps of a packet spread over many points: inside the 1e-6 bound
    assert np.max(np.abs(c32 - c64)) <= 1e-6, np.max(np.abs(c32 - c64))
    assert np.max(np.abs(p32 - p64)) <= 2e-4


def oracle_sod(oracle, np_, sh, sm, dt, nsteps, v, psi, absorb=0, vabc=None, quirks=0):
    p = oracle.make_prop(np_, dt, 0.0, nsteps * dt, sh, sm, lc=1, absorb=absorb, quirks=quirks)
    return oracle.psodfft(p, v, np.real(psi).copy(), np.imag(psi).copy(), vabc=vabc)


def gpu_sod(np_, sh, sm, dt, v, psi, nsteps, absorb=0, vabc=None, quirks=0):
    g = E.SodGrid(np_, sh, sm, dt, absorb=absorb, quirks=quirks)
    g.load(v, psi, vabc=vabc)
    g.run(nsteps)
    c, out = g.results()
    prev = g.previous()
    g.close()
    return c, out, prev


def close_until_overflow(got, ref, rtol=1e-9, lag=8):
    """C(t) of a run that overflows: |got - ref| <= rtol max(1, |ref|) wherever
    both are finite, got finite wherever ref is, and the first non-finite entry
    of got at most `lag` steps after ref's.  The GPU's kinetic factor carries
    the 1/N of the inverse transform before it (the reference divides after an
    unnormalised FFT), so its intermediates are N times smaller and overflow a
    few steps later."""
    got, ref = np.asarray(got), np.asarray(ref)
    fg, fr = np.isfinite(got), np.isfinite(ref)
    assert np.all(fg[fr])
    both = fg & fr
    rel = np.abs(got[both] - ref[both]) / np.maximum(1.0, np.abs(ref[both]))
    assert rel.max() <= rtol, rel.max()
    if not fr.all():
        first_r = np.argmin(fr)
        first_g = np.argmin(fg) if not fg.all() else len(fg)
        assert first_g - first_r <= lag, (first_r, first_g)


def test_golden_2d_sod_with_reference_defects(oracle):
    """The 32x32 coupled-Morse .PFSOD deck: with the reference's 2D kinetic
    table (dkeft.f:80-137) dt E_max is far above 1 and the executable's C(t)
    grows ~100x per step until it overflows; the GPU follows the oracle step
    by step relative to the growing magnitude, until the overflow."""
    case = G.setup_case("morse2d_sod")
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_NONE)
    c, psi, prev = gpu_sod(case["np"], case["sh"], case["sm"], case["dt"], case["vpot"],
                           case["psi"], ref["nc"] - 1, quirks=NAT.Q_SOD_SMOOTHW | NAT.Q_DIGT_ND)
    close_until_overflow(c, ref["c"])
    for got, r in ((psi, ref["u"] + 1j * ref["v"]), (prev, ref["u_prev"] + 1j * ref["v_prev"])):
        assert not np.isfinite(r).any() and not np.isfinite(got).any()
    gold = case["data"]["rows"]
    ok = np.isfinite(gold[:, 2])
    rel = np.abs(c.real[ok] - gold[ok, 2]) / np.maximum(1.0, np.abs(gold[ok, 2]))
    assert rel.max() < 1e-6


@pytest.mark.parametrize("np_,absorb,ref_smoothw", [
    ([64, 128], 0, False), ([128, 32], 1, False), ([64, 64], 2, False), ([64, 64], 2, True),
    ([32, 64, 32], 0, False), ([64, 32, 32], 2, True)])
def test_sod_nd_grids_match_oracle(oracle, np_, absorb, ref_smoothw):
    """SOD is stable only for dt * E_max < 1: dt = 5e-4 fs keeps the largest
    kinetic energy of these grids (128 points over 3 bohr) below that."""
    v, psi, sh, sm, grids = packet(np_, 3 * sum(np_))
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.02 * np.clip(grids[0] - 3.2, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 3.3, 0.97, 1.0).ravel(order="F")
    dt = 5e-4
    q_o = oracle.Q_SOD_SMOOTHW if ref_smoothw else 0
    q_g = NAT.Q_SOD_SMOOTHW if ref_smoothw else 0
    ref = oracle_sod(oracle, np_, sh, sm, dt, 150, v, psi, absorb=absorb, vabc=vabc, quirks=q_o)
    c, out, prev = gpu_sod(np_, sh, sm, dt, v, psi, ref["nc"] - 1, absorb=absorb, vabc=vabc,
                           quirks=q_g)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10


def test_sod_nd_continue_matches_one_run():
    v, psi, sh, sm, _ = packet([64, 64], 11)
    dt = 5e-4
    c1, p1, q1 = gpu_sod([64, 64], sh, sm, dt, v, psi, 120)
    g = E.SodGrid([64, 64], sh, sm, dt)
    g.load(v, psi)
    g.run(50)
    ca, _ = g.results()
    g.advance(70)
    cb, p2 = g.results()
    q2 = g.previous()
    g.close()
    assert np.max(np.abs(np.concatenate([ca, cb[1:]]) - c1)) <= 1e-12
    assert np.max(np.abs(p2 - p1)) <= 1e-12 and np.max(np.abs(q2 - q1)) <= 1e-12
