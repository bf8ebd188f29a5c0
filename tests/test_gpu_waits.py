"""Bounded device waits, exercised without any fault.

The SIL and PSOD kernels' grid barriers and the tensor-core GEMM's mbarrier
waits give up after a poll limit.  Here each wait is made to run out by a
flag that nothing sets -- a grid launch whose arrival count starts one short
(its first barrier can never complete), an mbarrier nobody arrives on -- with
a short limit; the kernels must return, report the time-out (error code,
INFO = 2 from the drop-in, the GEMM status word), and the device must stay
usable: the next run matches a clean run bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as N
from espec_b200 import fortran as F

pytestmark = pytest.mark.gpu


def _grid_case(n=64):
    x = np.linspace(0.5, 8.0, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    V = 0.17 * (1 - np.exp(-(X - 1.4))) ** 2 + 0.12 * (1 - np.exp(-1.2 * (Y - 1.8))) ** 2
    psi = np.exp(-((X - 1.6) ** 2 + (Y - 2.0) ** 2) / 0.045).astype(complex)
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2))
    h = x[1] - x[0]
    shm = [1.0 / (24 * 918 * h * h), 1.0 / (24 * 1500 * h * h)]
    return V.ravel(order="F"), psi.ravel(order="F"), shm


@pytest.fixture
def short_waits():
    lib = N.load()
    assert lib.espec_set_wait_limit(1 << 12) == 0
    yield lib
    lib.espec_selftest_short_arrivals(0)
    lib.espec_set_wait_limit(0)


@pytest.mark.parametrize("kind", ["sil", "psod"])
def test_grid_barrier_wait_gives_up_and_device_stays_usable(kind, short_waits):
    lib = short_waits
    v, psi, shm = _grid_case()

    def make():
        g = E.PsodGrid([64, 64], shm, 1e-4) if kind == "psod" else \
            E.SilGrid([64, 64], shm, 1e-3, 4)
        g.load(v, psi)
        return g

    g = make()
    g.run(5)
    c_ref, p_ref = g.results()
    g.close()

    assert lib.espec_selftest_short_arrivals(1) == 0
    g = make()
    g.run(5)
    with pytest.raises(E.EspecError, match="timed out"):
        g.results()
    g.close()

    g = make()
    g.run(5)
    c, p = g.results()
    g.close()
    assert np.array_equal(c, c_ref) and np.array_equal(p, p_ref)


def test_plnz_drop_in_returns_info_2_on_a_barrier_time_out(short_waits):
    lib = short_waits
    v, psi, shm = _grid_case()
    n = v.size
    dt = 1e-3

    def call():
        u, w = psi.real.copy(), psi.imag.copy()
        lnzvc = np.zeros((n, 16), order="F")
        info, _ = F.plnz(absorb=False, change=False, dim=".2D", prtcrl=".NO", tpabsor=".NONE",
                         lc=1, lmtreort=10, mp=4, mpi=14, mpr=13, mxdct=n, n=n, dt=dt, ti=0.0,
                         tf=4 * dt, tol=100.0, np_=[64, 64], shm=shm, vpot=v, vabc=None, u=u,
                         v=w, lnzvc=lnzvc)
        return info, u, w

    info0, u0, w0 = call()
    assert info0 in (0, 1)
    assert lib.espec_selftest_short_arrivals(1) == 0
    info, _, _ = call()
    assert info == 2
    info1, u1, w1 = call()
    assert info1 == info0 and np.array_equal(u1, u0) and np.array_equal(w1, w0)


def test_gemm_mbarrier_wait_gives_up():
    lib = N.load()
    st = C.c_int(-1)
    assert lib.espec_gemm_bf16_status(C.byref(st)) == 0  # clear
    gave_up = C.c_int(0)
    assert lib.espec_selftest_mbar_wait(1 << 10, C.byref(gave_up)) == 0
    assert gave_up.value == 1
    assert lib.espec_gemm_bf16_status(C.byref(st)) == 0
    assert st.value == 1
    assert lib.espec_gemm_bf16_status(C.byref(st)) == 0
    assert st.value == 0
