"""The benchmark configurations 2 and 3 themselves (not smaller stand-ins)
against the oracle: the 256 x 256 coupled-Morse grid with its quadratic
absorbing potential (split operator, CAP as .VOPTIC; SIL order 12, CAP as
the per-step mask exp(-W dt)), and the 128^3 anharmonic oscillator with its
edge CAP.  FP64 is held to 1e-10 against the oracle over the steps the
oracle finishes in seconds."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as N

pytestmark = pytest.mark.gpu

SHFS = 2.4188843243e-2


def _cap(q, strength=0.01, frac=0.15):
    lo, hi = q[0], q[-1]
    width = frac * (hi - lo)
    s = np.maximum(np.maximum(lo + width - q, q - (hi - width)), 0.0) / width
    return strength * s ** 2


def _c2():
    n = 256
    x = np.linspace(0.5, 8.0, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    morse = lambda q, de, a, re: de * (1 - np.exp(-a * (q - re))) ** 2  # noqa: E731
    V = morse(X, 0.17, 1.0, 1.4) + morse(Y, 0.12, 1.2, 1.8) + 0.01 * (X - 1.4) * (Y - 1.8)
    W = _cap(x)[:, None] + _cap(x)[None, :]
    psi = np.exp(-((X - 1.6) ** 2) / (2 * 0.15 ** 2) - ((Y - 2.0) ** 2) / (2 * 0.15 ** 2))
    psi = (psi / np.sqrt(np.sum(psi ** 2))).ravel(order="F").astype(complex)
    return n, x, V.ravel(order="F"), W.ravel(order="F"), psi


def test_config2_split_operator_with_cap_matches_oracle(oracle):
    n, x, v, w, psi = _c2()
    h = x[1] - x[0]
    dt = 1.0 * SHFS
    nsteps = 20
    p = oracle.make_prop([n, n], dt, 0.0, nsteps * dt, [h, h], [918.0, 1500.0], lc=1,
                         absorb=oracle.ABS_VOPTIC)
    ref = oracle.pspofft(p, v, psi.real.copy(), psi.imag.copy(), vabc=-w)
    nst = oracle.do_count(dt, nsteps * dt + dt, dt)
    g = E.SpoGrid([n, n], [h, h], [918.0, 1500.0], dt, absorb=N.ABS_VOPTIC)
    g.load(v, psi, vabc=-w)
    g.run(nst)
    c, out = g.results()
    g.close()
    assert np.max(np.abs(c - ref["c"])) <= 1e-10
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10


def test_config2_sil12_with_cap_mask_matches_oracle(oracle):
    n, x, v, w, psi = _c2()
    h = x[1] - x[0]
    dt = 1.0 * SHFS
    shm = [1.0 / (((24.0 * m) * h) * h) for m in (918.0, 1500.0)]
    mask = np.exp(-w * 1.0)
    nsteps = 4
    p = oracle.make_prop([n, n], dt, 0.0, nsteps * dt, [h, h], [918.0, 1500.0], lc=1, mp=12,
                         lmtreort=16, change=0, shm=shm, absorb=oracle.ABS_SMOOTHW)
    ref = oracle.plnz(p, v, psi.real.copy(), psi.imag.copy(), vabc=mask)
    nst = oracle.do_count(dt, nsteps * dt + dt, dt)
    g = E.SilGrid([n, n], shm, dt, 12, absorb=N.ABS_SMOOTHW)
    g.load(v, psi, vabc=mask)
    g.run(nst)
    c, out = g.results()
    g.close()
    assert np.max(np.abs(c - ref["c"])) <= 1e-10
    assert np.max(np.abs(out - (ref["u"] + 1j * ref["v"]))) <= 1e-10
