"""1D packets of sizes outside the register FFT plans (espec_b200/csrc/
spo1d_any.cu): any even N, FP64, with eSPec's mixed-radix FFT (fft3d.f)
behind them in the reference.  GPU against the oracle's restatement of
spofft.f / sodfft.f on the same inputs: |dC(t)| and |d psi| <= 1e-10, the same
bar as the register kernels; sizes with radices 2, 3, 4, 5, 7 and a large
prime factor (2 x 101), mixed in one batch with a register-plan size."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT
from espec_b200 import workloads as W

from test_gpu_spo1d import gpu_batch, oracle_batch, random_packets

pytestmark = pytest.mark.gpu

ANY = [250, 200, 202, 300, 490, 1000, 6000]


def test_spo_any_sizes_match_oracle(oracle):
    n, off, sh, sm, v, psi = random_packets(ANY + [256], seed=11)
    dt = 0.5 * W.SHFS
    c_ref, p_ref = oracle_batch(oracle, n, off, sh, sm, v, psi, dt, 300)
    c, p = gpu_batch(n, sh, sm, v, psi, dt, 300, "fp64")
    err = np.max(np.abs(c - c_ref), axis=1)
    assert np.max(err) <= 1e-10, dict(zip(n.tolist(), err))
    assert np.max(np.abs(p - p_ref)) <= 1e-10


def test_spo_any_size_reference_defect(oracle):
    """spofft.f:150-153 in-place kinetic multiply on a 250-point packet (the
    form the .PFSPO drop-in runs)."""
    n, off, sh, sm, v, psi = random_packets([250, 202], seed=12)
    dt = 0.005 * W.SHFS
    c_ref, p_ref = oracle_batch(oracle, n, off, sh, sm, v, psi, dt, 400,
                                quirks=oracle.Q_SPO_INPLACE)
    c, p = gpu_batch(n, sh, sm, v, psi, dt, 400, "fp64", quirks=NAT.Q_SPO_INPLACE)
    assert np.max(np.abs(c - c_ref)) <= 1e-10
    assert np.max(np.abs(p - p_ref)) <= 1e-10


@pytest.mark.parametrize("absorb", ["none", "voptic", "smoothw"])
def test_sod_any_sizes_match_oracle(oracle, absorb):
    from test_gpu_sod import oracle_sod, packet

    dt = 0.005 * W.SHFS
    sizes = [250, 300, 202]
    refs, packs = [], []
    for k, n in enumerate(sizes):
        x, sh, sm, v, psi = packet(n, 300 + k)
        xi, xf = x[0], x[-1]
        vabc, ab_o = None, 0
        if absorb == "voptic":
            vabc = oracle.absorbingbc([n], oracle.ABC_VOPTIC_POLIN, [1.6], [7.0], [sh], [xi],
                                      [xf], [-0.02, 2.0, 0.0])
            ab_o = oracle.ABS_VOPTIC
        elif absorb == "smoothw":
            vabc = oracle.absorbingbc([n], oracle.ABC_SMOOTHW, [1.0], [7.0], [sh], [xi], [xf],
                                      [0.05, 1.0, 0.0])
            ab_o = oracle.ABS_SMOOTHW
        refs.append(oracle_sod(oracle, n, sh, sm, v, psi, dt, 300, absorb=ab_o, vabc=vabc))
        packs.append((n, sh, sm, v, psi, vabc))
    nsteps = refs[0]["nc"] - 1
    ab_g = {"none": NAT.ABS_NONE, "voptic": NAT.ABS_VOPTIC, "smoothw": NAT.ABS_SMOOTHW}[absorb]
    b = E.SodBatch([p[0] for p in packs], [p[1] for p in packs], [p[2] for p in packs], dt,
                   absorb=ab_g)
    b.load(np.concatenate([p[3] for p in packs]), np.concatenate([p[4] for p in packs]),
           vabc=None if absorb == "none" else np.concatenate([p[5] for p in packs]))
    b.run(nsteps)
    c, psi = b.results()
    prev = b.previous()
    off = np.concatenate([[0], np.cumsum([p[0] for p in packs])])
    for k, r in enumerate(refs):
        assert np.max(np.abs(c[k] - r["c"])) <= 1e-10, (sizes[k], np.max(np.abs(c[k] - r["c"])))
        assert np.max(np.abs(psi[off[k]:off[k + 1]] - (r["u"] + 1j * r["v"]))) <= 1e-10
        assert np.max(np.abs(prev[off[k]:off[k + 1]] - (r["u_prev"] + 1j * r["v_prev"]))) <= 1e-10
    b.close()


def test_any_size_energies_match_oracle(oracle):
    """EFFT4 energy and norm of psi0 (the E column of the drop-in's table)."""
    n, off, sh, sm, v, psi = random_packets([250, 1000], seed=13)
    b = E.SpoBatch(n, sh, sm, 0.1 * W.SHFS, precision="fp64")
    b.load(v, psi)
    e, nrm = b.energies()
    for k in range(len(n)):
        sl = slice(off[k], off[k + 1])
        tc, bb = oracle.digt([int(n[k])], [sh[k]], [sm[k]])
        e_ref = oracle.efft4([int(n[k])], psi[sl], np.zeros(int(n[k])), tc, v[sl], bb)
        assert abs(e[k] - e_ref) <= 1e-12 * max(1.0, abs(e_ref)), (n[k], e[k], e_ref)
        assert abs(nrm[k] - np.sum(psi[sl] ** 2)) <= 1e-12
    b.close()

