"""The drop-ins' argument checks (ppsod_, pplnz_, and the time step of all), on the CPU: every
case here is refused with INFO = 2 and a reason on stderr before any device
work, and the caller's arrays are left as they were."""
import numpy as np
import pytest

from espec_b200 import fortran as F

N = 64


def common():
    return dict(absorb=False, dim=".1D", efc=".GAUS", prtcrl=".PARTIAL", tpabsor=".NONE", lc=1,
                mxdct=N, n=N, dt=0.01, ti=0.0, tf=0.1, tol=1.0, np_=[N], shm=[1.0], e0=1.0,
                tp=0.1, omg=1.0, dm=np.zeros(N), vpot=np.zeros(N), vabc=None)


CASES = [(dict(efc=".LASER"), "pulse"), (dict(dim=".4D"), "DIM"), (dict(n=N - 1), "N differs"),
         (dict(lc=0), "LC"), (dict(npr=7), "NPR"), (dict(dt=0.0), "DT"), (dict(dt=-0.01), "DT"),
         (dict(tf=1e12), "DT")]


@pytest.mark.parametrize("change,why", CASES)
def test_ppsod_refusals(capfd, change, why):
    lnzvc = np.zeros((N, 3), order="F")
    u1, v1 = np.ones(N), np.zeros(N)
    args = dict(common(), mpi=2, mpr=1, u1=u1, v1=v1, u2=np.zeros(N), v2=np.zeros(N),
                lnzvc=lnzvc)
    capfd.readouterr()
    assert F.ppsod(**dict(args, **change)) == 2
    err = capfd.readouterr()[1]
    assert err.startswith("espec_gpu PPSOD:") and why in err, err
    assert not lnzvc.any() and (u1 == 1).all() and not v1.any()


@pytest.mark.parametrize("change,why", CASES + [(dict(mp=20, lmtreort=30), "order")])
def test_pplnz_refusals(capfd, change, why):
    lnzvc = np.zeros((N, 14), order="F")
    u, v = np.ones(N), np.zeros(N)
    args = dict(common(), change=True, lmtreort=10, mp=10, mpi=12, mpr=11, u=u, v=v, lnzvc=lnzvc)
    capfd.readouterr()
    info, mp = F.pplnz(**dict(args, **change))
    assert info == 2
    err = capfd.readouterr()[1]
    assert err.startswith("espec_gpu PPLNZ:") and why in err, err
    assert not lnzvc.any() and (u == 1).all() and not v.any()


@pytest.mark.parametrize("dt,tf", [(0.0, 0.1), (-0.01, 0.1), (0.01, 1e12)])
def test_time_step_refused_by_every_dropin(capfd, dt, tf):
    """DT <= 0, or more than 1e9 steps: INFO = 2 from PSPOFFT, PSODFFT, PLNZ
    and PSOD too, before any device work."""
    z = np.zeros(N)
    base = dict(absorb=False, dim=".1D", prtcrl=".PARTIAL", tpabsor=".NONE", lc=1, mpi=3, mpr=2,
                mxdct=N, n=N, dt=dt, ti=0.0, tf=tf, tol=1.0, np_=[N], vpot=z, vabc=None)
    lnzvc = np.zeros((N, 12), order="F")
    capfd.readouterr()
    assert F.pspofft(**base, sh=[0.01], sm=[1000.0], u1=np.ones(N), v1=np.zeros(N),
                     tc=np.zeros(N), lnzvc=lnzvc) == 2
    assert F.psodfft(**base, sh=[0.01], sm=[1000.0], u1=np.ones(N), v1=np.zeros(N),
                     u2=np.zeros(N), v2=np.zeros(N), tc=np.zeros(N), lnzvc=lnzvc) == 2
    info, _ = F.plnz(**dict(base, mpi=12, mpr=11), change=True, lmtreort=10, mp=10, shm=[1.0],
                     u=np.ones(N), v=np.zeros(N), lnzvc=lnzvc)
    assert info == 2
    assert F.psod(**base, shm=[1.0], u1=np.ones(N), v1=np.zeros(N), u2=np.zeros(N),
                  v2=np.zeros(N), lnzvc=lnzvc) == 2
    err = capfd.readouterr()[1]
    assert err.count("DT must be positive") == 4, err
    assert not lnzvc.any()
