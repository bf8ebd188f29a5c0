"""The GPU kernels against the shipped eSPec executable itself.

The fixtures are the executable's printed partial C(t) tables (F10.7) for the
1D Morse decks of tests/golden/make_golden.py; the GPU FP64 forms, run with
the reference's defect switches where the executable has them, must agree
to print precision at every printed step."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT

import golden_cases as G

pytestmark = pytest.mark.gpu

PRINT = 1.01e-7


def _gpu_c(case, nsteps):
    meta = case["meta"]
    absorb = {0: NAT.ABS_NONE, 1: NAT.ABS_VOPTIC, 2: NAT.ABS_SMOOTHW}[case["absorb"]]
    if meta["prop"] == ".PFSPO":
        b = E.SpoBatch(case["np"], case["sh"], case["sm"], case["dt"], precision="fp64",
                       absorb=absorb, quirks=NAT.Q_SPO_INPLACE)
    else:
        b = E.SodBatch(case["np"], case["sh"], case["sm"], case["dt"], absorb=absorb,
                       quirks=NAT.Q_SOD_SMOOTHW)
    b.load(case["vpot"], case["psi"], vabc=case["vabc"])
    b.run(nsteps)
    c, _ = b.results()
    b.close()
    return c[0]


@pytest.mark.parametrize("name", ["morse1d_spo", "morse1d_spo_voptic", "morse1d_spo_smooth",
                                  "morse1d_sod", "morse1d_sod_voptic", "morse1d_sod_smooth"])
def test_gpu_reproduces_executable(name):
    case = G.setup_case(name)
    rows = case["data"]["rows"]  # one printed row per step (LC = 1)
    c = _gpu_c(case, rows.shape[0] - 1)
    assert c.shape[0] == rows.shape[0]
    d = np.max(np.abs(np.stack([c.real, c.imag], 1) - rows[:, 2:4]))
    assert d <= PRINT, d
