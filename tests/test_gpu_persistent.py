"""The persistent launch (one kernel over every packet size, items claimed
from a device counter, longest first) against the per-class launches.

Both shapes run the same plans and tables per size (the persistent kernel
uses each size's default variant), so C(t) and psi(TF) must be bit for bit
the same; the FP64 form is also checked against the oracle.
"""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run(w, precision, launch, nsteps=None, split=None):
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
    b.set_launch(launch)
    b.load(w["vpot"], w["psi"])
    ns = w["nsteps"] if nsteps is None else nsteps
    if split:
        b.run(split)
        c1, _ = b.results()
        b.advance(ns - split)
        c2, p = b.results()
        c = np.concatenate([c1, c2[:, 1:]], axis=1)
    else:
        b.run(ns)
        c, p = b.results()
    b.close()
    return c, p


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_equals_per_class_launches(precision):
    # uneven counts: partial items in several classes
    w = W.morse_scan(npk=203, nsteps=150, seed=11)
    c_p, p_p = _run(w, precision, "persistent")
    c_c, p_c = _run(w, precision, "classes")
    assert np.array_equal(c_p, c_c)
    assert np.array_equal(p_p, p_c)


def test_persistent_fp64_matches_oracle(oracle):
    w = W.morse_scan(npk=37, nsteps=200, seed=12)
    c, p = _run(w, "fp64", "persistent")
    c_ref, u, v = oracle.spo_batch(w["off"], w["sh"], w["sm"], w["vpot"], w["psi"],
                                   np.zeros_like(w["psi"]), w["dt_fs"], w["nsteps"], nthreads=8)
    assert np.max(np.abs(c - c_ref)) <= 1e-10
    assert np.max(np.abs(p - (u + 1j * v))) <= 1e-10


def test_persistent_resumed_run_equals_one_run():
    w = W.morse_scan(npk=40, nsteps=120, seed=13)
    c1, p1 = _run(w, "fp64", "persistent")
    c2, p2 = _run(w, "fp64", "persistent", split=50)
    # the resumed run re-applies the half V phase to the stored psi
    assert np.max(np.abs(c1 - c2)) <= 1e-12
    assert np.max(np.abs(p1 - p2)) <= 1e-12


def test_persistent_shape_refused_for_4096_point_packets():
    w = W.morse_scan(npk=2, nsteps=10, seed=14, sizes=(4096,))
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="fp64")
    with pytest.raises(E.EspecError):
        b.set_launch("persistent")
    b.close()


@pytest.mark.parametrize("launch", ["persistent", "classes"])
def test_nonfinite_packets_are_counted(launch):
    """A packet whose potential holds a NaN propagates NaN into C(t); the
    device counts it (once), the other packets stay finite."""
    w = W.morse_scan(npk=20, nsteps=30, seed=15)
    v = w["vpot"].copy()
    v[w["off"][3] + 5] = np.nan
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="fp64")
    b.set_launch(launch)
    b.load(v, w["psi"])
    b.run(w["nsteps"])
    assert b.nonfinite() == 1
    c, _ = b.results()
    assert not np.all(np.isfinite(c[3])) and np.all(np.isfinite(np.delete(c, 3, axis=0)))
    b.load(w["vpot"], w["psi"])
    b.run(w["nsteps"])
    assert b.nonfinite() == 0
    b.close()
