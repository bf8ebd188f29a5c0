"""GPU parity of the finite-difference second-order-differences propagator
(.PSOD: psod.f, sod.f, au1d.f/au2di.f/au3d.f) against the oracle's
restatement, FP64: |dC(t)|, |dpsi(TF)|, |dpsi(TF - dt)| <= 1e-10; against the
shipped executable's printed C(t) at its print precision."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT

import golden_cases as G

pytestmark = pytest.mark.gpu


def gpu_psod(np_, shm, dt, v, psi, nsteps, absorb=0, vabc=None, quirks=0, ctas=None):
    g = E.PsodGrid(np_, shm, dt, absorb=absorb, quirks=quirks)
    if ctas:
        g.set_ctas(ctas)
    g.load(v, psi, vabc=vabc)
    g.run(nsteps)
    c, out = g.results()
    prev = g.previous()
    g.close()
    return c, out, prev


@pytest.mark.parametrize("name", ["morse1d_psod", "morse1d_psod_voptic", "morse1d_psod_smooth",
                                  "morse2d_psod"])
def test_psod_golden_decks(oracle, name):
    case = G.setup_case(name)
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_NONE)
    assert case["lc"] == 1
    c, psi, prev = gpu_psod(case["np"], case["shm"], case["dt"], case["vpot"], case["psi"],
                            ref["nc"] - 1, absorb=case["absorb"], vabc=case["vabc"],
                            quirks=NAT.Q_PSOD_COPY)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(psi - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10
    gold = case["data"]["rows"]
    assert np.max(np.abs(c.real - gold[:, 2])) <= 1.01e-7
    assert np.max(np.abs(c.imag - gold[:, 3])) <= 1.01e-7


def packet(np_, seed):
    rng = np.random.default_rng(seed)
    axes = [np.linspace(-1.0, 1.0, n) * (0.6 + 0.2 * a) for a, n in enumerate(np_)]
    grids = np.meshgrid(*axes, indexing="ij")
    v = sum(0.5 * (0.8 + 0.3 * a) * g ** 2 for a, g in enumerate(grids)) + 0.05 * grids[0] ** 3
    psi = np.exp(-sum((g - 0.1 * (a + 1)) ** 2 / 0.08 for a, g in enumerate(grids)))
    psi = psi * np.exp(1j * (3.0 * grids[0] - 1.5 * grids[-1] + 0.2 * rng.standard_normal()))
    psi = psi / np.sqrt(np.sum(np.abs(psi) ** 2))
    sh = [ax[1] - ax[0] for ax in axes]
    return v.ravel(order="F"), psi.ravel(order="F"), sh, grids


@pytest.mark.parametrize("np_,absorb,quirk", [
    ([301], 0, False), ([301], 0, True), ([257], 1, False), ([256], 2, True),
    ([40, 36], 0, True), ([48, 33], 1, False), ([40, 40], 2, False),
    ([12, 10, 8], 0, False), ([9, 7, 11], 1, True), ([10, 12, 9], 2, False)])
def test_psod_random_grids(oracle, np_, absorb, quirk):
    """Complex initial states, so the restart-copy defect (psod.f:136-141) shows
    when it is switched on; dt such that dt E_max < 1 on every grid."""
    v, psi, sh, grids = packet(np_, sum(np_) + absorb)
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.05 * np.clip(grids[0] - 0.3, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F")
    dt = 0.002 * NAT.SHFS
    q_o = oracle.Q_PSOD_COPY if quirk else 0
    p = oracle.make_prop(np_, dt, 0.0, 120 * dt, sh, sm, lc=1, absorb=absorb, quirks=q_o,
                         shm=shm)
    ref = oracle.psod(p, v, np.real(psi), np.imag(psi), vabc=vabc)
    c, out, prev = gpu_psod(np_, shm, dt, v, psi, ref["nc"] - 1, absorb=absorb, vabc=vabc,
                            quirks=NAT.Q_PSOD_COPY if quirk else 0)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10


@pytest.mark.parametrize("np_,dt_au,absorb", [([1024, 640], 2e-4, 0), ([1024, 640], 2e-4, 1),
                                               ([2048, 600], 2e-4, 2),
                                               ([700000], 5e-10, 2), ([100, 96, 64], 0.01, 1)])
def test_psod_large_grids(oracle, np_, dt_au, absorb):
    """Grids of 16 or more points per thread, where the plan takes every
    co-resident CTA (two per SM) instead of one per SM: the same
    results as the oracle; dt below the SOD limit 1 / E_max of each grid."""
    v, psi, sh, grids = packet(np_, 3 + absorb)
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.05 * np.clip(grids[0] - 0.3, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F")
    dt = dt_au * NAT.SHFS
    p = oracle.make_prop(np_, dt, 0.0, 8 * dt, sh, sm, lc=1, absorb=absorb, shm=shm)
    ref = oracle.psod(p, v, np.real(psi), np.imag(psi), vabc=vabc)
    c, out, prev = gpu_psod(np_, shm, dt, v, psi, ref["nc"] - 1, absorb=absorb, vabc=vabc)
    assert np.isfinite(ref["c"]).all()
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10


def test_psod_continue_and_energies(oracle):
    np_ = [64, 48]
    v, psi, sh, _ = packet(np_, 9)
    sm = [918.0, 1500.0]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dt = 0.002 * NAT.SHFS
    c1, p1, q1 = gpu_psod(np_, shm, dt, v, psi, 90)
    g = E.PsodGrid(np_, shm, dt)
    g.load(v, psi)
    e0, n0 = g.energies()
    ref_e = oracle.eigenerg(np_, shm, v, psi.real) + oracle.eigenerg(np_, shm, v, psi.imag)
    assert abs(e0 - ref_e) <= 1e-12 * abs(ref_e) and abs(n0 - 1.0) <= 1e-12
    g.run(33)
    ca, _ = g.results()
    g.advance(57)
    cb, p2 = g.results()
    q2 = g.previous()
    e1, n1 = g.energies()
    g.close()
    assert np.max(np.abs(np.concatenate([ca, cb[1:]]) - c1)) <= 1e-12
    assert np.max(np.abs(p2 - p1)) <= 1e-12 and np.max(np.abs(q2 - q1)) <= 1e-12
    ref_e1 = oracle.eigenerg(np_, shm, v, p2.real) + oracle.eigenerg(np_, shm, v, p2.imag)
    assert abs(e1 - ref_e1) <= 1e-12 * abs(ref_e1)
    assert abs(n1 - np.sum(np.abs(p2) ** 2)) <= 1e-12


@pytest.mark.parametrize("np_,ctas,absorb,quirk", [
    ([300, 70], 4, 0, True), ([300, 70], 4, 1, False), ([512, 80], 4, 2, True),
    ([260, 100], 6, 0, False), ([301, 70], 4, 1, True), ([257, 64], 2, 2, False)])
def test_psod_column_strips(oracle, np_, ctas, absorb, quirk):
    """The column-strip pass of 2D grids (CTA count a multiple of the strip
    count, 16 or more rows per band), forced on small grids by the CTA count,
    ragged last strip included: the oracle's results, the restart-copy
    defect and the absorbers as on the point-range pass, for even and odd
    nx and one or several bands."""
    v, psi, sh, grids = packet(np_, 17 + absorb)
    sm = [1000.0, 1400.0]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.05 * np.clip(grids[0] - 0.3, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F")
    dt = 0.0005 * NAT.SHFS
    q_o = oracle.Q_PSOD_COPY if quirk else 0
    p = oracle.make_prop(np_, dt, 0.0, 40 * dt, sh, sm, lc=1, absorb=absorb, quirks=q_o,
                         shm=shm)
    ref = oracle.psod(p, v, np.real(psi), np.imag(psi), vabc=vabc)
    c, out, prev = gpu_psod(np_, shm, dt, v, psi, ref["nc"] - 1, absorb=absorb, vabc=vabc,
                            quirks=NAT.Q_PSOD_COPY if quirk else 0, ctas=ctas)
    assert np.max(np.abs(c - ref["c"])) <= 1e-10, np.max(np.abs(c - ref["c"]))
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(prev - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10
