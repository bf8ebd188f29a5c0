"""The drop-ins print the partial auto-correlation table in the reference's
Fortran formats (pspofft.f:147-148).  Pinned against the text the shipped
executable printed (tests/golden/*_partial.txt): every row, re-formatted
from its parsed values by the library, must come out byte for byte."""
import os

import numpy as np
import pytest

from espec_b200 import fortran

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["morse1d_spo", "morse1d_sod", "morse1d_spo_voptic"]
HEAD = [" ", " Partial auto-correlation function:", " ==================================", "",
        "       *t/fs*       *E/a.u.*        *Cr(t)*       *Ci(t)*      *|C(t)|*      *|C|*"]


def golden_text(case):
    with open(os.path.join(GOLDEN, case + "_partial.txt")) as f:
        return f.read().split("\n")[:-1]


@pytest.mark.parametrize("case", CASES)
def test_rows_reformat_byte_for_byte(case):
    lines = golden_text(case)
    assert lines[:5] == HEAD
    rows = lines[5:]
    assert len(rows) == 200
    for line in rows:
        vals = [float(x) for x in line.split()]
        assert fortran.format_crl_row(*vals) == line + "\n", line


def test_first_row():
    row = fortran.format_crl_row(0.0, 0.0261122, 1.0, 0.0, 1.0, 1.0)
    assert row == ("     0.00000000   0.261122E-01     1.0000000     0.0000000    1.00000000"
                   "    1.000000\n")


def test_negative_small_and_overflow():
    row = fortran.format_crl_row(-1e-12, -0.5, -1e-9, -0.99999999, 12.5, 1.5)
    t, e, cr, ci, ct, fn = (row[1:15], row[18:30], row[34:44], row[48:58], row[62:72],
                            row[76:84])
    assert t == "   -0.00000000"
    assert e == "-.500000E+00"
    assert cr == "-0.0000000"
    assert ci == "-1.0000000"
    assert ct == "**********"
    assert fn == "1.500000"
    assert len(row) == 85


def test_exponent_and_nonfinite():
    row = fortran.format_crl_row(0.0, 1.25e-120, np.nan, np.inf, -np.inf, 0.0)
    assert row[18:30] == "0.125000-119"
    assert row[34:44].strip() == "NaN"
    assert row[48:58].strip() == "Infinity"
    assert row[62:72].strip() == "-Infinity"
