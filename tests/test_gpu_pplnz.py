"""The pplnz_ drop-in (SUBROUTINE PPLNZ, pplnz.f) against the oracle's
restatement and the executable: the printed table (T, E with and without the
field, Cr, Ci, |C|^2, the populations, the norm) to half a unit of every
printed digit, LNZVC's C(t) rows and psi(TF) to 1e-10, INFO, LNZ's order
messages, MP, VPOT as CHPOT leaves it, and the last Lanczos basis."""
import os

import numpy as np
import pytest

from espec_b200 import _native as NAT
from espec_b200 import fortran as F
from espec_b200 import grid as GR

import golden_cases as G
from test_gpu_ppsod import EFC, PRT, PULSES, check_rows, table
from test_gpu_psod import packet

pytestmark = pytest.mark.gpu


def expected_head(dim, npr):
    title = " Auto-correlation function:" if dim == ".1D" else " Partial auto-correlation function:"
    groups = ["*|P%d|^2*" % (i - 1) for i in range(1, npr + 1)] + ["*|c0|^2*"]
    h = "        *t/fs*     *ET/a.u.*      *E0/a.u.*      *Pr(t)*    *Pi(t)*   "
    return [" ", title, " ==================================", "", h + "   ".join(groups)]


def run_case(oracle, capfd, np_, shape, par, mask, npr, lc, prtcrl, mp, lmt=10, change=True,
             tf=0.2, tol=1e-3):
    v, psi, sh, grids = packet(np_, sum(np_) + 5 * npr + lc + mp)
    n = int(np.prod(np_))
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    dm = (0.8 * grids[0] + 0.3 * grids[0] ** 2).ravel(order="F")
    vabc = np.where(grids[0] > 0.35, 0.97, 1.0).ravel(order="F") if mask else None
    absorb = NAT.ABS_SMOOTHW if mask else NAT.ABS_NONE
    nw = max(npr - 1, 0)
    rng = np.random.default_rng(n + npr)
    w = []
    for k in range(nw):
        c = rng.uniform(-0.2, 0.3, len(np_))
        g = np.exp(-sum((gr - c[a]) ** 2 / 0.1 for a, gr in enumerate(grids))).ravel(order="F")
        w.append(g / np.sqrt(np.sum(g * g)))
    w = np.array(w).reshape(nw, n)
    # dt E_max below 1 on these grids: with sil.f's cos-before-sin a larger
    # step grows the norm without bound
    dt, ti = 0.005 * NAT.SHFS, 0.0
    p = oracle.make_prop(np_, dt, ti, tf, sh, sm, lc=lc, absorb=absorb, prtcrl=PRT[prtcrl],
                         tol=tol, shm=shm, mp=mp, lmtreort=lmt, change=int(change),
                         quirks=oracle.Q_SIL_INPLACE)
    ref = oracle.pplnz_table(p, v, dm, shape, par, npr, w, np.real(psi), np.imag(psi), vabc=vabc)
    ef = GR.pplnz_field(shape, par, ti, tf, dt)
    m = lmt if (change and mp > lmt) else mp
    mpr, mpi = m + 1, m + 2  # C(t) after the Lanczos basis, as espec.f lays LNZVC out
    kp = m + 2               # W_k = LNZVC(., KP+k): past both
    mxdct = max(n, len(ef) // lc + 8)
    lnzvc = np.zeros((mxdct, kp + nw + 1), order="F")
    for k in range(nw):
        lnzvc[:n, kp + k] = w[k]
    u, vv = np.ascontiguousarray(psi.real), np.ascontiguousarray(psi.imag)
    vpot = np.array(v)
    p6 = list(par) + [0.0] * (6 - len(par))
    t0, td = (0.0, p6[3]) if shape == NAT.PULSE_SIN2 else (p6[3], 0.0)
    dim = ".%dD" % len(np_)
    capfd.readouterr()
    info, mp_out = F.pplnz(absorb=mask, change=change, dim=dim, efc=EFC[shape], prtcrl=prtcrl,
                           tpabsor=".SMOOTHW" if mask else ".NONE", lc=lc, lmtreort=lmt, mp=mp,
                           mpi=mpi, mpr=mpr, mxdct=mxdct, n=n, dt=dt, ti=ti, tf=tf, tol=tol,
                           np_=np_, shm=shm, e0=p6[0], tp=p6[1], omg=p6[2], t0=t0, td=td,
                           sni=p6[4], kl=int(p6[5]), npr=npr, kp=kp, dm=dm, vpot=vpot, vabc=vabc,
                           u=u, v=vv, lnzvc=lnzvc)
    out, err = capfd.readouterr()
    assert err == ""
    return dict(ref=ref, ef=ef, v=v, dm=dm, w=w, n=n, m=m, kp=kp, info=info, mp=mp_out, out=out,
                lnzvc=lnzvc, u=u, vv=vv, vpot=vpot, dim=dim)


@pytest.mark.parametrize("np_,pulse,mask,npr,lc,prtcrl,mp", [
    ([301], "gaus", False, 0, 1, ".PARTIAL", 10), ([256], "ggaus", True, 3, 3, ".PARTIAL", 8),
    ([300], "sin2", False, 1, 2, ".YES", 12), ([40, 36], "gaus", False, 4, 1, ".PARTIAL", 8),
    ([48, 33], "sin2", True, 6, 4, ".YES", 6), ([10, 12, 9], "gaus", True, 2, 5, ".NO", 6)])
def test_pplnz_dropin_matches_oracle(oracle, capfd, np_, pulse, mask, npr, lc, prtcrl, mp):
    shape, par = PULSES[pulse]
    r = run_case(oracle, capfd, np_, shape, par, mask, npr, lc, prtcrl, mp)
    ref, n, m = r["ref"], r["n"], r["m"]
    assert r["info"] == ref["info"]
    if prtcrl == ".NO":
        assert r["out"] == ""
    else:
        lines = r["out"].split("\n")
        kept = [l for l in lines if not l.startswith((" Error NREORT", " NREORT=", " Modifing"))]
        assert (len(kept) < len(lines)) == (mp > 10)  # LNZ's messages when MP > LMTREORT
        head, rows = table("\n".join(kept), 6 + npr)
        assert head == expected_head(r["dim"], npr)
        check_rows(rows, ref["rows"])
    nc = ref["nc"]
    c = r["lnzvc"][:nc, m] + 1j * r["lnzvc"][:nc, m + 1]
    first = 0 if prtcrl != ".NO" else 1  # LNZVC(1, .) is written inside the print test only
    assert np.max(np.abs(c[first:] - ref["c"][first:])) <= 1e-10
    if first:
        assert c[0] == 0
    assert not r["lnzvc"][nc:, m:m + 2].any()
    for k in range(max(npr - 1, 0)):  # the projection vectors are read, not written
        assert np.array_equal(r["lnzvc"][:n, r["kp"] + k], r["w"][k])
    assert np.max(np.abs(r["u"] + 1j * r["vv"] - (ref["u"] + 1j * ref["v"]))) <= 1e-10
    np.testing.assert_array_equal(r["vpot"], r["v"] - r["dm"] * r["ef"][-1])
    # LNZVC(., 1..MP): the last step's Lanczos basis, orthonormal
    basis = r["lnzvc"][:n, :m]
    assert np.max(np.abs(basis.T @ basis - np.eye(m))) < 1e-8
    assert r["mp"] == m


@pytest.mark.parametrize("change", [True, False])
def test_pplnz_dropin_order_messages(oracle, capfd, change):
    """MP = 12 > LMTREORT = 10: LNZ's messages between the rows -- once,
    with MP lowered for good, under *CHANGE; twice per step (both chains)
    without it -- as in PLNZ (lnz.f:64-72)."""
    shape, par = PULSES["gaus"]
    r = run_case(oracle, capfd, [256], shape, par, False, 0, 2, ".PARTIAL", 12, change=change,
                 tf=0.1)
    out = r["out"]
    nsteps = len(r["ef"]) - 1
    msgs = out.count(" Error NREORT > LMTREORT\n")
    assert msgs == (1 if change else 2 * nsteps)
    assert ("Modifing NREORT to correct value!" in out) == change
    assert r["mp"] == (10 if change else 12)
    lines = out.split("\n")
    k = lines.index(" Error NREORT > LMTREORT")
    assert lines[k - 1].split()[0] == "0.000000"  # after the first row, before the second
    kept = [l for l in lines if not l.startswith((" Error NREORT", " NREORT=", " Modifing"))]
    head, rows = table("\n".join(kept), 6)
    check_rows(rows, r["ref"]["rows"])


def test_pplnz_dropin_info_on_drift(oracle, capfd):
    """INFO = 1 when a printed row's norm drifts from the first row's
    beyond TOL percent, without an absorber (pplnz.f:270-274)."""
    shape, par = PULSES["gaus"]
    r = run_case(oracle, capfd, [256], shape, par, False, 0, 1, ".PARTIAL", 10, tol=1e-12)
    assert r["ref"]["info"] == r["info"] == 1
    r = run_case(oracle, capfd, [256], shape, par, False, 0, 1, ".PARTIAL", 10, tol=1.0)
    assert r["ref"]["info"] == r["info"] == 0
    r = run_case(oracle, capfd, [256], shape, par, True, 0, 1, ".PARTIAL", 10, tol=1e-12)
    assert r["ref"]["info"] == r["info"] == 0


def test_pplnz_dropin_rejects(capfd):
    n = 64
    lnzvc = np.zeros((n, 14), order="F")
    z = np.zeros(n)
    args = dict(absorb=False, change=True, dim=".1D", efc=".GAUS", prtcrl=".PARTIAL",
                tpabsor=".NONE", lc=1, lmtreort=10, mp=10, mpi=12, mpr=11, mxdct=n, n=n, dt=0.01,
                ti=0.0, tf=0.1, tol=1.0, np_=[n], shm=[1.0], e0=1.0, tp=0.1, omg=1.0, dm=z,
                vpot=np.zeros(n), vabc=None, u=np.ones(n), v=np.zeros(n), lnzvc=lnzvc)
    capfd.readouterr()
    assert F.pplnz(**dict(args, efc=".LASER"))[0] == 2
    assert "pulse" in capfd.readouterr()[1]
    assert F.pplnz(**dict(args, dim=".4D"))[0] == 2
    assert F.pplnz(**dict(args, npr=7))[0] == 2
    assert F.pplnz(**dict(args, mp=20, lmtreort=30))[0] == 2
    assert F.pplnz(**dict(args, n=n - 1))[0] == 2
    assert not lnzvc.any()


@pytest.mark.parametrize("name,npr", [("deck_ppsil", 0), ("deck_ppsil_proj", 2)])
def test_pplnz_dropin_matches_executable(capfd, name, npr):
    """The .PPSIL decks of tests/golden/deck_ppsil* (Gaussian pulse, .EXP
    dipole mu(R) = 0.5 R exp(-0.3 R), MP = 10; the _proj deck with NPR = 2,
    KP = 0 after rdinput.f:659, its projection vector LNZVC(., 1) zero as in
    the executable): the drop-in prints the executable's table head and rows
    (one printed unit, plus 4e-7 in Cr, Ci, |C|^2 for the reference's
    ABSTOL = 1e-6 eigenvalue bisection)."""
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
    lnzvc = np.zeros((n, 12), order="F")
    capfd.readouterr()
    info, mp = F.pplnz(absorb=False, change=True, dim=".1D", efc=".GAUS", prtcrl=".PARTIAL",
                       tpabsor=".NONE", lc=2, lmtreort=10, mp=10, mpi=12, mpr=11, mxdct=n, n=n,
                       dt=dt, ti=0.0, tf=256 * dt, tol=1e3, np_=[n], shm=[G.shm_of(918.0, sh)],
                       e0=5.0e7, tp=0.1, omg=2.5, t0=0.15, sni=0.0, npr=npr, kp=0, dm=dm,
                       vpot=np.array(v), vabc=None, u=np.array(psi), v=np.zeros(n), lnzvc=lnzvc)
    out, err = capfd.readouterr()
    assert err == "" and info == 0 and mp == 10
    text = open(os.path.join(G.GOLDEN, name, "expected.txt")).read()
    ncol = 6 + npr
    gh, gold = table(text, ncol)
    head, rows = table(out, ncol)
    assert head == gh
    assert rows.shape == gold.shape == (129, ncol)
    d_ = np.abs(rows - gold)
    unit = np.array([1e-6, 0, 0, 1e-5, 1e-5] + [1e-6] * (ncol - 5))
    slack = np.zeros(ncol)
    slack[3:5] = 4e-7
    if npr:
        slack[5] = 4e-7
    num = [0] + list(range(3, ncol))
    assert np.all(d_[:, num] <= (unit * 1.01 + slack)[num]), d_.max(axis=0)
    e_unit = 10.0 ** (np.floor(np.log10(np.abs(gold[:, 1:3]))) - 5)
    assert np.all(d_[:, 1:3] <= e_unit * 1.01)
    got_lines = [l for l in out.split("\n") if len(l.split()) == ncol and l.split()[0][0].isdigit()]
    gold_lines = [l for l in text.split("\n") if len(l.split()) == ncol and l.split()[0][0].isdigit()]
    assert sum(a == b for a, b in zip(got_lines, gold_lines)) >= 0.8 * len(gold_lines)
