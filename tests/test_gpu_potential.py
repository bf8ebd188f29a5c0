"""GPU analytic potentials (POT1D/POT2D/POT3D on GVPOT's grid loop) against
the oracle's restatement of potfuncs.f / gvpot.f, every form, with and
without the shift by the grid minimum."""
import numpy as np
import pytest

from espec_b200 import potential as P
from espec_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORMS_1D = {
    ".OHS": [1.7, 0.08], ".DOHS": [1.7, 0.08, 2.5, 3.0, 0.01], ".MORSEM": [1.6, 1.1, 0.17],
    ".ANTI-MORSEM": [1.6, 1.1, 0.17], ".MOD-MORSE": [1.6, 1.1, 0.17, 0.9, 0.02],
    ".MORSE": [1.4, 1.0, 0.17], ".ANTI-MORSE": [1.4, 1.0, 0.17],
    ".DMORSE": [1.5, 2.5, 0.2, 1.2, 0.05, 3.0], ".STEP": [1.0, 4.0, 0.3],
    ".BARRIER": [2.0, 2.4, 0.05], ".CONST": [0.07]}
LEPS = [1.4, 1.0, 0.17, 1.5, 1.1, 0.16, 1.45, 1.05, 0.15, 0.1, 0.12, 0.08, 1.9]
FORMS_2D = {
    ".OHS": [1.7, 0.08, 2.0, 0.05], ".MORSE": [1.4, 1.0, 0.17, 1.8, 1.2, 0.12],
    ".LSM": [1.4, 1.0, 0.17, 1.2, 0.15, 1.8, 1.1], ".LS": [1.4, 1.0, 0.17, 1.2, 0.15],
    ".LBH_CC": [0.3, 0.6, 0.17, 1.1, 1.6], ".LBH": [0.3, 0.6, 0.17, 1.1, 1.6],
    ".LEPS_CC": LEPS, ".LEPS": LEPS, ".WELLXY": [1.0, 4.0, 0.3, 1.5, 5.0, 0.2],
    ".WELLX": [1.0, 4.0, 0.3], ".WELLY": [1.5, 5.0, 0.2], ".WELL": [1.0, 4.0, 1.5, 5.0, 0.4],
    ".BARRIERXY": [2.0, 2.4, 0.05, 3.0, 3.3, 0.02], ".BARRIERX": [2.0, 2.4, 0.05],
    ".BARRIERY": [3.0, 3.3, 0.02], ".BARRIER": [2.0, 2.4, 3.0, 3.3, 0.05], ".CONST": [0.07]}
FORMS_3D = {".OHS": [1.7, 0.08, 2.0, 0.05, 1.9, 0.06], ".STEP": [1.0, 4.0, 1.5, 5.0, 1.2, 4.5, 0.3],
            ".BARRIER": [2.0, 2.4, 1.0, 4.0, 1.5, 5.0, 0.05], ".LEPS": LEPS, ".CONST": [0.07]}


def _close(a, b):
    # the reference's formulas overflow on parts of some grids (.LS's 1/(2(RY -
    # CST(1))) term): the same non-finite values at the same points, the
    # finite ones to 1e-13
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return False
    if not np.array_equal(a[~fb], b[~fb], equal_nan=True):
        return False
    return not fb.any() or np.max(np.abs(a[fb] - b[fb]) / np.maximum(1.0, np.abs(b[fb]))) <= 1e-13


@pytest.mark.parametrize("shiftp", [False, True])
@pytest.mark.parametrize("name", sorted(FORMS_1D))
def test_gvpot_1d_batch_matches_oracle(oracle, name, shiftp):
    rng = np.random.default_rng(5)
    npts = rng.choice([256, 384, 1000, 2048], size=9).astype(np.int32)
    xi = rng.uniform(0.4, 0.8, 9)
    sh = 7.5 / (npts - 1)
    cst = np.array([np.asarray(FORMS_1D[name]) * rng.uniform(0.9, 1.1) for _ in range(9)])
    v, xmin = P.gvpot_1d(npts, xi, sh, name, cst, shiftp=shiftp)
    v = v.cpu().numpy()
    off = np.concatenate([[0], np.cumsum(npts)])
    for k in range(9):
        ref, xm = oracle.gvpot(shiftp, name, [int(npts[k])], [xi[k]], [sh[k]], cst[k])
        assert _close(v[off[k]:off[k + 1]], ref), (name, k)
        if shiftp:
            assert xmin[k] == xm


@pytest.mark.parametrize("shiftp", [False, True])
@pytest.mark.parametrize("name", sorted(FORMS_2D))
def test_gvpot_2d_matches_oracle(oracle, name, shiftp):
    np_, xi, sh, sm = [96, 80], [0.6, 0.9], [0.05, 0.06], [1.0, 1.2, 1.4]
    ref, _ = oracle.gvpot(shiftp, name, np_, xi, sh, FORMS_2D[name], sm=sm)
    v = P.gvpot_nd(np_, xi, sh, name, FORMS_2D[name], sm=sm, shiftp=shiftp).cpu().numpy()
    assert _close(v, ref)


@pytest.mark.parametrize("quirk", [0, 64])
@pytest.mark.parametrize("name", sorted(FORMS_3D))
def test_gvpot_3d_matches_oracle(oracle, name, quirk):
    np_, xi, sh = [32, 24, 20], [0.6, 0.9, 1.0], [0.12, 0.15, 0.2]
    ref, _ = oracle.gvpot(True, name, np_, xi, sh, FORMS_3D[name], quirk3d=quirk)
    v = P.gvpot_nd(np_, xi, sh, name, FORMS_3D[name], shiftp=True, quirks=quirk).cpu().numpy()
    assert _close(v, ref)


def test_scan_potentials_built_on_the_gpu_equal_the_workload():
    """The 4096-packet Morse scan's potentials from its parameter table."""
    w = W.morse_scan()
    p = w["params"]
    cst = np.stack([p["re"], p["a"], p["de"]], axis=1)
    v, _ = P.gvpot_1d(w["n"], np.full(w["npk"], 0.5), w["sh"], ".MORSE", cst, shiftp=False)
    assert np.max(np.abs(v.cpu().numpy() - w["vpot"])) <= 1e-12
