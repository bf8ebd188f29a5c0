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
    assert np.max(np.abs(c32 - c64)) <= 2e-5, np.max(np.abs(c32 - c64))
    assert np.max(np.abs(p32 - p64)) <= 2e-4
