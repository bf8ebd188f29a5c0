"""CPU checks of the analytic potentials: the name -> form mapping of the
library (the reference's prefix tests, potfuncs.f), and the oracle's GVPOT
(gvpot.f) against closed forms and its shift rules."""
import numpy as np
import pytest

from espec_b200 import potential as P
from espec_b200 import workloads as W


@pytest.mark.parametrize("nd,name,kind", [
    (1, ".MORSEM", 3), (1, ".MORSE", 6), (1, ".MORSEX", 6), (1, ".ANTI-MORSEM", 4),
    (1, ".ANTI-MORSE", 7), (1, ".MOD-MORSE", 5), (1, ".FREE", 11), (1, ".BOGUS", 0),
    (2, ".LSM", 12), (2, ".LS", 13), (2, ".LBH_CC", 14), (2, ".LEPS_CC", 16), (2, ".WELLXY", 18),
    (2, ".BARRIERX", 23), (2, ".BARRIER", 10), (3, ".LEPS", 17), (3, ".MORSE", 0)])
def test_pot_kind_follows_the_reference_prefix_order(nd, name, kind):
    assert P.pot_kind(name, nd) == kind


def test_oracle_gvpot_morse_equals_closed_form(oracle):
    x0, n, de, a, re = 0.5, 512, 0.17, 1.1, 1.4
    sh = 7.5 / (n - 1)
    v, xmin = oracle.gvpot(False, ".MORSE", [n], [x0], [sh], [re, a, de])
    x = x0 + np.arange(n) * sh
    assert np.max(np.abs(v - W.morse(x, de, a, re))) <= 1e-15


def test_oracle_gvpot_shift_rules(oracle):
    # 1D: shifted only when the minimum is above 1e-6 (gvpot.f:27)
    v, xmin = oracle.gvpot(True, ".OHS", [64], [-1.0], [0.05], [0.3, 2.0])
    assert abs(v.min()) < 1e-15 and abs(xmin - (-1.0 + 26 * 0.05)) < 1e-12
    v0, _ = oracle.gvpot(True, ".CONST", [16], [0.0], [0.1], [-0.5])
    assert np.all(v0 == -0.5)  # a negative minimum is kept in 1D
    # 2D: shifted when |minimum| > 1e-6 (gvpot.f:64)
    v2, _ = oracle.gvpot(True, ".CONST", [8, 8], [0.0, 0.0], [0.1, 0.1], [-0.5], sm=[1.0, 1.0])
    assert np.all(v2 == 0.0)
