"""The ppsod_ drop-in (SUBROUTINE PPSOD, ppsod.f) against the oracle's
restatement and the executable: the printed table (T, E with and without the
field, Cr, Ci, |C|^2, the populations |<W_k|psi>|^2, the norm) to half a unit
of every printed digit, LNZVC's C(t) rows, psi(TF) and psi(TF - dt) to 1e-10,
INFO, and VPOT as CHPOT leaves it."""
import os

import numpy as np
import pytest

from espec_b200 import _native as NAT
from espec_b200 import fortran as F
from espec_b200 import grid as GR

import golden_cases as G
from test_gpu_psod import packet

pytestmark = pytest.mark.gpu

EFC = {NAT.PULSE_GAUS: ".GAUS", NAT.PULSE_GGAUS: ".GGAUS", NAT.PULSE_SIN2: ".SIN2",
       NAT.PULSE_NONE: ".NONE"}
TPABSOR = {0: ".NONE", 1: ".VOPTIC", 2: ".SMOOTHW"}
PRT = {".YES": 2, ".PARTIAL": 1, ".NO": 0}
# FORMAT 1021 (ppsod.f): F14.6, 2 x E12.6 (ET, E0), 2 x F8.5, then F8.6
UNIT = [1e-6, None, None, 1e-5, 1e-5]
PULSES = {"gaus": (NAT.PULSE_GAUS, (6e7, 0.08, 2.5, 0.12, 0.3)),
          "ggaus": (NAT.PULSE_GGAUS, (3e11, 0.08, 2.5, 0.12, 0.3, 2)),
          "sin2": (NAT.PULSE_SIN2, (6e7, 0.2, 3.0, 0.05, 0.0))}


def table(out, ncol):
    """The head lines and the numeric rows of a PPSOD table on stdout."""
    lines = out.split("\n")
    i = [k for k, l in enumerate(lines) if l in (" Auto-correlation function:",
                                                  " Partial auto-correlation function:")][0]
    head = lines[i - 1:i + 4]
    rows = []
    for l in lines[i + 4:]:
        f = l.split()
        if len(f) != ncol:
            break
        rows.append([float(x) for x in f])
    return head, np.array(rows).reshape(-1, ncol)


def check_rows(got, ref, units=0.5):
    """Each printed number lies within half a unit of its last digit of the
    oracle's exact value (plus 1e-9 for the GPU/oracle difference); one unit
    between two printed tables."""
    assert got.shape == ref.shape, (got.shape, ref.shape)
    for j in range(got.shape[1]):
        if j in (1, 2):
            unit = 10.0 ** (np.floor(np.log10(np.abs(ref[:, j]))) - 5)
        else:
            unit = UNIT[j] if j < len(UNIT) else 1e-6
        err = np.abs(got[:, j] - ref[:, j])
        assert np.all(err <= units * unit * 1.001 + 1e-9), (j, np.max(err / unit))


def expected_head(dim, npr, kp, nispg):
    title = " Auto-correlation function:" if dim == ".1D" else " Partial auto-correlation function:"
    fmt = "%2d" if npr + kp - 1 > 10 else "%1d"
    groups = ["*|P" + fmt % (nispg - 1) + "|^2*"]
    groups += ["*|P" + fmt % (i - 1 + kp) + "|^2*" for i in range(1, npr + 1)]
    groups += [" |c" + fmt % (nispg - 1) + "|^2 "]
    h = "        *t/fs*     *ET/a.u.*      *E0/a.u.*      *Pr(t)*    *Pi(t)*   "
    return [" ", title, " ==================================", "", h + "   ".join(groups)]


def run_case(oracle, capfd, np_, shape, par, absorb, npr, lc, prtcrl, tf=0.25, kp=2, tol=1e-3):
    v, psi, sh, grids = packet(np_, sum(np_) + 3 * npr + lc)
    n = int(np.prod(np_))
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dm = (0.8 * grids[0] + 0.3 * grids[0] ** 2).ravel(order="F")
    vabc = None
    if absorb == NAT.ABS_VOPTIC:
        vabc = -0.05 * np.clip(grids[0] - 0.3, 0, None).ravel(order="F") ** 2
    elif absorb == NAT.ABS_SMOOTHW:
        vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F")
    # projection vectors: real Gaussians at shifted centres, normalised
    rng = np.random.default_rng(n + npr)
    w = []
    for k in range(npr):
        c = rng.uniform(-0.2, 0.3, len(np_))
        g = np.exp(-sum((gr - c[a]) ** 2 / 0.1 for a, gr in enumerate(grids))).ravel(order="F")
        w.append(g / np.sqrt(np.sum(g * g)))
    w = np.array(w).reshape(npr, n)
    dt, ti = 0.002 * NAT.SHFS, 0.0
    p = oracle.make_prop(np_, dt, ti, tf, sh, sm, lc=lc, absorb=absorb, prtcrl=PRT[prtcrl],
                         tol=tol, shm=shm)
    ref = oracle.ppsod_table(p, v, dm, shape, par, w, np.real(psi), np.imag(psi), vabc=vabc)
    ef = GR.ppsod_field(shape, par, ti, tf, dt)
    mxdct = max(n, len(ef) // lc + 8)
    lnzvc = np.zeros((mxdct, kp + npr + 1), order="F")
    for k in range(npr):
        lnzvc[:n, kp + k] = w[k]
    u1, v1 = np.ascontiguousarray(psi.real), np.ascontiguousarray(psi.imag)
    u2, v2 = np.zeros(n), np.zeros(n)
    vpot = np.array(v)
    p6 = list(par) + [0.0] * (6 - len(par))
    t0, td = (0.0, p6[3]) if shape == NAT.PULSE_SIN2 else (p6[3], 0.0)
    dim = ".%dD" % len(np_)
    capfd.readouterr()
    info = F.ppsod(absorb=absorb != 0, dim=dim, efc=EFC[shape], prtcrl=prtcrl,
                   tpabsor=TPABSOR[absorb], lc=lc, mpi=2, mpr=1, mxdct=mxdct, n=n, dt=dt, ti=ti,
                   tf=tf, tol=tol, np_=np_, shm=shm, e0=p6[0], tp=p6[1], omg=p6[2], t0=t0,
                   td=td, sni=p6[4], kl=int(p6[5]), npr=npr, kp=kp, dm=dm, vpot=vpot,
                   vabc=vabc, u1=u1, v1=v1, u2=u2, v2=v2, lnzvc=lnzvc)
    out, err = capfd.readouterr()
    assert err == ""
    return dict(ref=ref, ef=ef, v=v, dm=dm, w=w, n=n, kp=kp, info=info, out=out, lnzvc=lnzvc,
                u1=u1, v1=v1, u2=u2, v2=v2, vpot=vpot, dim=dim)


@pytest.mark.parametrize("np_,pulse,absorb,npr,lc,prtcrl", [
    ([301], "gaus", 0, 0, 1, ".PARTIAL"), ([256], "ggaus", 1, 2, 3, ".PARTIAL"),
    ([300], "sin2", 2, 1, 2, ".YES"), ([40, 36], "gaus", 0, 3, 1, ".PARTIAL"),
    ([48, 33], "sin2", 1, 6, 4, ".YES"), ([10, 12, 9], "gaus", 0, 2, 5, ".NO")])
def test_ppsod_dropin_matches_oracle(oracle, capfd, np_, pulse, absorb, npr, lc, prtcrl):
    shape, par = PULSES[pulse]
    r = run_case(oracle, capfd, np_, shape, par, absorb, npr, lc, prtcrl)
    ref, n = r["ref"], r["n"]
    assert r["info"] == ref["info"]
    if prtcrl == ".NO":
        assert r["out"] == ""
    else:
        head, rows = table(r["out"], 7 + npr)
        assert head == expected_head(r["dim"], npr, r["kp"], 1)
        check_rows(rows, ref["rows"])
    nc = ref["nc"]
    c = r["lnzvc"][:nc, 0] + 1j * r["lnzvc"][:nc, 1]
    first = 0 if prtcrl != ".NO" else 1  # LNZVC(1, .) is written inside the print test only
    assert np.max(np.abs(c[first:] - ref["c"][first:])) <= 1e-10
    if first:
        assert c[0] == 0
    assert not r["lnzvc"][nc:, :2].any()
    for k in range(npr):  # the projection vectors are read, not written
        assert np.array_equal(r["lnzvc"][:n, r["kp"] + k], r["w"][k])
    assert np.max(np.abs(r["u2"] + 1j * r["v2"] - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    assert np.max(np.abs(r["u1"] + 1j * r["v1"] - (ref["u_prev"] + 1j * ref["v_prev"]))) <= 1e-10
    np.testing.assert_array_equal(r["vpot"], r["v"] - r["dm"] * r["ef"][-1])


def test_ppsod_dropin_info_on_drift(oracle, capfd):
    """INFO = 1 when the norm of a printed loop row drifts beyond TOL percent
    without an absorber (ppsod.f:440-444); never with one."""
    shape, par = PULSES["gaus"]
    r = run_case(oracle, capfd, [256], shape, par, 0, 0, 1, ".PARTIAL", tf=0.1, tol=1e-8)
    assert r["ref"]["info"] == r["info"] == 1
    r = run_case(oracle, capfd, [256], shape, par, 0, 0, 1, ".PARTIAL", tf=0.1, tol=1e-6)
    assert r["ref"]["info"] == r["info"] == 0
    r = run_case(oracle, capfd, [256], shape, par, 1, 0, 1, ".PARTIAL", tf=0.1, tol=1e-8)
    assert r["ref"]["info"] == r["info"] == 0


def test_ppsod_dropin_rejects(capfd):
    n = 64
    lnzvc = np.zeros((n, 3), order="F")
    z = np.zeros(n)
    args = dict(absorb=False, dim=".1D", efc=".GAUS", prtcrl=".PARTIAL", tpabsor=".NONE", lc=1,
                mpi=2, mpr=1, mxdct=n, n=n, dt=0.01, ti=0.0, tf=0.1, tol=1.0, np_=[n], shm=[1.0],
                e0=1.0, tp=0.1, omg=1.0, dm=z, vpot=np.zeros(n), vabc=None, u1=np.ones(n),
                v1=np.zeros(n), u2=np.zeros(n), v2=np.zeros(n), lnzvc=lnzvc)
    capfd.readouterr()
    assert F.ppsod(**dict(args, efc=".LASER")) == 2
    assert "pulse" in capfd.readouterr()[1]
    assert F.ppsod(**dict(args, dim=".4D")) == 2
    assert F.ppsod(**dict(args, npr=7)) == 2
    assert F.ppsod(**dict(args, absorb=True, tpabsor=".CAP")) == 2
    assert F.ppsod(**dict(args, n=n - 1)) == 2
    assert not lnzvc.any()


def test_ppsod_dropin_matches_executable(capfd):
    """The .PPSOD deck of tests/golden/deck_ppsod (Gaussian pulse, .EXP dipole
    mu(R) = 0.5 R exp(-0.3 R)): the drop-in prints the executable's table head
    and rows."""
    d = os.path.join(G.GOLDEN, "deck_ppsod")
    lines = open(os.path.join(d, "wf_pot.inp")).read().split("\n")
    n = 256
    x = np.array([float(l.split()[0]) for l in lines[1:1 + n]])
    psi = np.array([float(l.split()[1]) for l in lines[1:1 + n]])
    v = np.array([float(l.split()[1]) for l in lines[2 + n:2 + 2 * n]])
    sh = (x[-1] - x[0]) / (n - 1)
    dt = 0.05 * 2.4188843243e-2
    r_ab = x[0] + np.arange(n) * sh  # dipl.f:62-66
    dm = 0.5 * r_ab * np.exp(-0.3 * r_ab)
    lnzvc = np.zeros((n, 2), order="F")
    capfd.readouterr()
    info = F.ppsod(absorb=False, dim=".1D", efc=".GAUS", prtcrl=".PARTIAL", tpabsor=".NONE", lc=2,
                   mpi=2, mpr=1, mxdct=n, n=n, dt=dt, ti=0.0, tf=256 * dt, tol=1e3, np_=[n],
                   shm=[G.shm_of(918.0, sh)], e0=5.0e7, tp=0.1, omg=2.5, t0=0.15, sni=0.0,
                   dm=dm, vpot=np.array(v), vabc=None, u1=np.array(psi), v1=np.zeros(n),
                   u2=np.zeros(n), v2=np.zeros(n), lnzvc=lnzvc)
    out, err = capfd.readouterr()
    assert err == "" and info == 0
    text = open(os.path.join(d, "expected.txt")).read()
    gh, gold = table(text, 7)
    head, rows = table(out, 7)
    assert head == gh
    assert rows.shape == gold.shape
    got_lines = [l for l in out.split("\n") if len(l.split()) == 7 and l.split()[0][0].isdigit()]
    gold_lines = [l for l in text.split("\n") if len(l.split()) == 7 and l.split()[0][0].isdigit()]
    same = sum(a == b for a, b in zip(got_lines, gold_lines))
    assert same >= 0.9 * len(gold_lines), same
    check_rows(rows, gold, units=1.0)
