"""GPU parity of the batched SOD-FFT propagator (.PFSOD) against the oracle's
restatement of psodfft.f/sodfft.f: FP64, |dC(t)| <= 1e-10."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT
from espec_b200 import workloads as W

pytestmark = pytest.mark.gpu

SOD_SIZES = [256, 384, 512, 768, 1024, 1536, 2048]


def oracle_sod(oracle, n, sh, sm, v, psi, dt, nsteps, absorb=0, vabc=None, quirks=0):
    p = oracle.make_prop([n], dt, 0.0, nsteps * dt, [sh], [sm], lc=1, absorb=absorb, quirks=quirks)
    r = oracle.psodfft(p, v, psi, np.zeros(n), vabc=vabc)
    return r


def packet(n, seed):
    rng = np.random.default_rng(seed)
    x0, x1 = 0.5, 8.0
    sh = (x1 - x0) / (n - 1)
    x = x0 + np.arange(n) * sh
    v = W.morse(x, rng.uniform(0.05, 0.25), rng.uniform(0.6, 1.6), rng.uniform(1.0, 2.5))
    psi = W.gaussian(x, rng.uniform(1.2, 2.5), rng.uniform(0.1, 0.3))
    return x, sh, rng.uniform(900.0, 30000.0), v, psi


def test_sod_all_sizes_match_oracle(oracle):
    dt = 0.005 * W.SHFS  # SOD is stable only for dt * E_max < 1
    refs, packs = [], []
    for k, n in enumerate(SOD_SIZES):
        x, sh, sm, v, psi = packet(n, 100 + k)
        r = oracle_sod(oracle, n, sh, sm, v, psi, dt, 300)
        refs.append(r)
        packs.append((n, sh, sm, v, psi))
    nsteps = refs[0]["nc"] - 1
    assert all(r["nc"] - 1 == nsteps for r in refs)
    b = E.SodBatch([p[0] for p in packs], [p[1] for p in packs], [p[2] for p in packs], dt)
    b.load(np.concatenate([p[3] for p in packs]), np.concatenate([p[4] for p in packs]))
    b.run(nsteps)
    c, psi = b.results()
    prev = b.previous()
    off = np.concatenate([[0], np.cumsum([p[0] for p in packs])])
    for k, r in enumerate(refs):
        assert np.max(np.abs(c[k] - r["c"])) <= 1e-10, (SOD_SIZES[k], np.max(np.abs(c[k] - r["c"])))
        assert np.max(np.abs(psi[off[k]:off[k + 1]] - (r["u"] + 1j * r["v"]))) <= 1e-10
        assert np.max(np.abs(prev[off[k]:off[k + 1]] - (r["u_prev"] + 1j * r["v_prev"]))) <= 1e-10
    b.close()


@pytest.mark.parametrize("kind", ["voptic", "smoothw", "smoothw_reference"])
def test_sod_absorbers_match_oracle(oracle, kind):
    n = 1024
    x, sh, sm, v, psi = packet(n, 7)
    sm = 918.0
    xi, xf = x[0], x[-1]
    dt = 0.005 * W.SHFS
    q_o = q_g = 0
    if kind == "voptic":
        vabc = oracle.absorbingbc([n], oracle.ABC_VOPTIC_POLIN, [1.6], [2.2], [sh], [xi], [xf],
                                  [-0.02, 2.0, 0.0])
        ab_o, ab_g = oracle.ABS_VOPTIC, NAT.ABS_VOPTIC
    else:
        vabc = oracle.absorbingbc([n], oracle.ABC_SMOOTHW, [1.55], [2.3], [sh], [xi], [xf],
                                  [0.05, 1.0, 0.0])
        ab_o, ab_g = oracle.ABS_SMOOTHW, NAT.ABS_SMOOTHW
        if kind == "smoothw_reference":
            q_o, q_g = oracle.Q_SOD_SMOOTHW, NAT.Q_SOD_SMOOTHW
    r = oracle_sod(oracle, n, sh, sm, v, psi, dt, 400, absorb=ab_o, vabc=vabc, quirks=q_o)
    b = E.SodBatch([n], [sh], [sm], dt, absorb=ab_g, quirks=q_g)
    b.load(v, psi, vabc=vabc)
    b.run(r["nc"] - 1)
    c, p = b.results()
    b.close()
    assert np.max(np.abs(c[0] - r["c"])) <= 1e-10
    assert np.max(np.abs(p - (r["u"] + 1j * r["v"]))) <= 1e-10
