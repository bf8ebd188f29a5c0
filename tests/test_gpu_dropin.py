"""GPU parity of the Fortran drop-ins pspofft_/psodfft_ (PSPOFFT pspofft.f:1-150,
PSODFFT psodfft.f:1-211) and of the plan calls they are built from
(espec_prop_continue, espec_prop_energies).

Each drop-in call is compared with the oracle's restatement of the same
subroutine on the same inputs: LNZVC columns, psi(TF), TC and INFO (FP64,
|d| <= 1e-10), and the printed partial auto-correlation table, row by row,
with the rows the shipped executable printed (tests/golden) at its print
precision."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import fortran as F
from espec_b200 import workloads as W

import golden_cases as G

pytestmark = pytest.mark.gpu

CASES = ["morse1d_spo", "morse1d_spo_voptic", "morse1d_spo_smooth",
         "morse1d_sod", "morse1d_sod_voptic", "morse1d_sod_smooth"]
TPABSOR = {None: ".NONE", "VOPTIC_POLIN": ".VOPTIC_POLIN", "SMOOTHW": ".SMOOTHW"}


def parse_table(out):
    lines = out.split("\n")
    i = lines.index(" Partial auto-correlation function:")
    assert lines[i - 1] == " " and lines[i + 1].startswith(" ====") and lines[i + 2] == ""
    assert lines[i + 3].split() == ["*t/fs*", "*E/a.u.*", "*Cr(t)*", "*Ci(t)*", "*|C(t)|*",
                                    "*|C|*"]
    rows, text = [], []
    for l in lines[i + 4:]:
        if len(l.split()) != 6:
            break
        text.append(l)
        rows.append([float(x) for x in l.split()])
    return np.array(rows), text


def call_dropin(case, prtcrl, lc=None, tol=None, mxdct=None, ncols=4, mpr=2, mpi=3, tf=None):
    m = case["meta"]
    n = case["np"][0]
    lc = case["lc"] if lc is None else lc
    tf = case["tf"] if tf is None else tf
    nsteps = 2 * int(round((tf - case["ti"]) / case["dt"])) + 4
    mxdct = nsteps // lc + 4 if mxdct is None else mxdct
    lnzvc = np.zeros((mxdct, ncols), order="F")
    u1 = np.array(case["psi"], dtype=np.float64)
    v1 = np.zeros(n)
    tc = np.zeros(n)
    args = dict(absorb=case["absorb"] != 0, dim=".1D", prtcrl=prtcrl,
                tpabsor=TPABSOR[m.get("absorb")], lc=lc, mpi=mpi, mpr=mpr, mxdct=mxdct, n=n,
                dt=case["dt"], ti=case["ti"], tf=tf, tol=case["tol"] if tol is None else tol,
                np_=case["np"], sh=case["sh"], sm=case["sm"], u1=u1, v1=v1, tc=tc,
                vpot=case["vpot"], vabc=case["vabc"], lnzvc=lnzvc)
    if m["prop"] == ".PFSPO":
        info = F.pspofft(**args)
        return dict(info=info, u=u1, v=v1, tc=tc, lnzvc=lnzvc)
    u2, v2 = np.zeros(n), np.zeros(n)
    info = F.psodfft(u2=u2, v2=v2, **args)
    return dict(info=info, u=u2, v=v2, u_prev=u1, v_prev=v1, tc=tc, lnzvc=lnzvc)


def oracle_of(case, prtcrl, lc=None, tol=None, tf=None):
    c = dict(case)
    if lc is not None:
        c["lc"] = lc
    if tol is not None:
        c["tol"] = tol
    if tf is not None:
        c["tf"] = tf
    return G.run_oracle(c, case["ref_quirks"], prtcrl=prtcrl)


def check_arrays(case, got, ref, mpr=2, mpi=3):
    nc = ref["nc"]
    col = got["lnzvc"]
    assert np.max(np.abs(col[:nc, mpr - 1] - ref["c"].real)) <= 1e-10
    assert np.max(np.abs(col[:nc, mpi - 1] - ref["c"].imag)) <= 1e-10
    assert not np.any(col[nc:, [mpr - 1, mpi - 1]]), "samples past NC written"
    others = [j for j in range(col.shape[1]) if j not in (mpr - 1, mpi - 1)]
    assert not np.any(col[:, others]), "other LNZVC columns touched"
    assert np.max(np.abs(got["u"] - ref["u"])) <= 1e-10
    assert np.max(np.abs(got["v"] - ref["v"])) <= 1e-10
    if "u_prev" in got:
        assert np.max(np.abs(got["u_prev"] - ref["u_prev"])) <= 1e-10
        assert np.max(np.abs(got["v_prev"] - ref["v_prev"])) <= 1e-10
    tc_ref = E.spo.digt_1d(case["np"][0], case["sh"][0], case["sm"][0])
    assert np.array_equal(got["tc"], tc_ref)
    assert got["info"] == ref["info"]


@pytest.mark.parametrize("name", CASES)
def test_dropin_matches_oracle_and_executable(oracle, capfd, name):
    case = G.setup_case(name)
    capfd.readouterr()
    got = call_dropin(case, ".PARTIAL")
    out, err = capfd.readouterr()
    assert err == ""
    ref = oracle_of(case, oracle.PRT_PARTIAL)
    check_arrays(case, got, ref)
    rows, text = parse_table(out)
    # against the oracle's rows (FP64 values, then printed): within print precision
    assert rows.shape == ref["rows"].shape
    half_ulp = np.array([5e-9, 0, 5e-8, 5e-8, 5e-9, 5e-7])
    d = np.abs(rows - ref["rows"])
    assert np.all(d[:, [0, 2, 3, 4, 5]] <= half_ulp[[0, 2, 3, 4, 5]] + 1e-10)
    # E12.6 keeps 6 significant digits
    e_ulp = 10.0 ** (np.floor(np.log10(np.abs(ref["rows"][:, 1]))) - 5)
    assert np.all(np.abs(rows[:, 1] - ref["rows"][:, 1]) <= 0.5 * e_ulp * 1.001)
    # against the executable's printed rows: the same text except where the
    # last printed digit rounds the other way
    gold = case["data"]["rows"]
    assert rows.shape == gold.shape
    ulp = np.array([1e-8, 0, 1e-7, 1e-7, 1e-8, 1e-6])
    dg = np.abs(rows - gold)
    assert np.all(dg[:, [0, 2, 3, 4, 5]] <= ulp[[0, 2, 3, 4, 5]] * 1.01)
    assert np.all(np.abs(rows[:, 1] - gold[:, 1]) <= e_ulp * 1.01)
    if name in ("morse1d_spo", "morse1d_sod", "morse1d_spo_voptic"):
        with open(f"{G.GOLDEN}/{name}_partial.txt") as f:
            golden_lines = f.read().split("\n")[5:5 + 150]
        same = sum(a == b for a, b in zip(text[:150], golden_lines))
        assert same >= 140, same


@pytest.mark.parametrize("name", ["morse1d_spo", "morse1d_sod_voptic"])
def test_dropin_stride_columns_and_no_print(oracle, capfd, name):
    case = G.setup_case(name)
    tf = 300 * case["dt"]
    capfd.readouterr()
    got = call_dropin(case, ".NO", lc=7, ncols=8, mpr=5, mpi=6, tf=tf)
    out, _ = capfd.readouterr()
    assert out == ""
    ref = oracle_of(case, oracle.PRT_NONE, lc=7, tf=tf)
    check_arrays(case, got, ref, mpr=5, mpi=6)
    # '.PARTIAL' with LC = 7 prints the rows of steps 0, 7, 14, ...
    got = call_dropin(case, ".PARTIAL", lc=7, ncols=8, mpr=5, mpi=6, tf=tf)
    out, _ = capfd.readouterr()
    ref = oracle_of(case, oracle.PRT_PARTIAL, lc=7, tf=tf)
    check_arrays(case, got, ref, mpr=5, mpi=6)
    rows, _ = parse_table(out)
    assert rows.shape == ref["rows"].shape
    assert np.max(np.abs(rows[:, [0, 2, 3]] - ref["rows"][:, [0, 2, 3]])) <= 5.1e-8


@pytest.mark.parametrize("name", ["morse1d_spo", "morse1d_spo_voptic", "morse1d_sod",
                                  "morse1d_sod_voptic"])
def test_dropin_info_drift_semantics(oracle, capfd, name):
    """INFO = 1 on drift: PSPOFFT tests the norm only with an absorber
    (pspofft.f:137-142), PSODFFT only without one (psodfft.f:178-183)."""
    case = G.setup_case(name)
    tf = 200 * case["dt"]
    for tol in (1e-12, 1e-7, 1e-3, 10.0):
        got = call_dropin(case, ".YES", tol=tol, tf=tf)
        ref = oracle_of(case, oracle.PRT_YES, tol=tol, tf=tf)
        assert got["info"] == ref["info"], (tol, got["info"], ref["info"])
    capfd.readouterr()


def test_dropin_rejects_what_it_does_not_run(capfd):
    case = G.setup_case("morse1d_spo")
    capfd.readouterr()
    n = case["np"][0]
    lnzvc = np.zeros((8, 3), order="F")
    u1, v1, tc = np.array(case["psi"]), np.zeros(n), np.zeros(n)
    info = F.pspofft(absorb=False, dim=".4D", prtcrl=".NO", tpabsor=".NONE", lc=1, mpi=3, mpr=2,
                     mxdct=8, n=n, dt=case["dt"], ti=0.0, tf=case["dt"], tol=1.0, np_=[n],
                     sh=case["sh"], sm=case["sm"], u1=u1, v1=v1, tc=tc, vpot=case["vpot"],
                     vabc=None, lnzvc=lnzvc)
    _, err = capfd.readouterr()
    assert info == 2 and "DIM" in err
    assert np.array_equal(u1, case["psi"]) and not lnzvc.any()


def test_continue_and_energies_match_single_run(oracle):
    """A run split by espec_prop_continue follows the same trajectory as one
    run; energies/norms of the state match the oracle's EFFT4 and norm."""
    rng = np.random.default_rng(5)
    sizes = [384, 1024, 2048]
    packs = []
    for n in sizes:
        x0, x1 = 0.5, 8.0
        sh = (x1 - x0) / (n - 1)
        x = x0 + np.arange(n) * sh
        v = W.morse(x, rng.uniform(0.05, 0.25), rng.uniform(0.6, 1.6), rng.uniform(1.0, 2.5))
        psi = W.gaussian(x, rng.uniform(1.2, 2.5), rng.uniform(0.1, 0.3)) * np.exp(0.3j * x)
        packs.append((n, sh, rng.uniform(900.0, 30000.0), v, psi))
    dt = 0.01 * W.SHFS
    vcat = np.concatenate([p[3] for p in packs])
    pcat = np.concatenate([p[4] for p in packs])
    off = np.concatenate([[0], np.cumsum(sizes)])
    for cls, kw in [(E.SpoBatch, dict(precision="fp64")), (E.SpoBatch, dict(precision="mixed")),
                    (E.SodBatch, {})]:
        tol = 2e-6 if kw.get("precision") == "mixed" else 1e-11
        one = cls(sizes, [p[1] for p in packs], [p[2] for p in packs], dt, **kw)
        one.load(vcat, pcat)
        e0, n0 = one.energies()
        for k, (n, sh, sm, v, psi) in enumerate(packs):
            tcr = E.spo.digt_1d(n, sh, sm)
            ref_e = oracle.efft4([n], psi.real, psi.imag, tcr, v, 1.0 / n)
            assert abs(e0[k] - ref_e) <= 1e-12 * abs(ref_e)
            assert abs(n0[k] - np.sum(np.abs(psi) ** 2)) <= 1e-12
        one.run(90)
        c_one, psi_one = one.results()
        seg = cls(sizes, [p[1] for p in packs], [p[2] for p in packs], dt, **kw)
        seg.load(vcat, pcat)
        seg.run(30)
        c_a, _ = seg.results()
        seg.advance(1)
        c_b, _ = seg.results()
        seg.advance(59)
        c_c, psi_seg = seg.results()
        c_seg = np.concatenate([c_a, c_b[:, 1:], c_c[:, 1:]], axis=1)
        assert np.max(np.abs(c_seg - c_one)) <= tol, (cls, kw)
        assert np.max(np.abs(psi_seg - psi_one)) <= tol
        e1, n1 = seg.energies()
        for k, (n, sh, sm, v, psi) in enumerate(packs):
            p = psi_seg[off[k]:off[k + 1]]
            tcr = E.spo.digt_1d(n, sh, sm)
            ref_e = oracle.efft4([n], p.real.copy(), p.imag.copy(), tcr, v, 1.0 / n)
            assert abs(e1[k] - ref_e) <= 1e-12 * abs(ref_e)
            assert abs(n1[k] - np.sum(np.abs(p) ** 2)) <= 1e-12
        one.close()
        seg.close()


# ---------------------------------------------------------------------------
# PLNZ (plnz.f:1-155)
# ---------------------------------------------------------------------------
def call_plnz(case, prtcrl, mp=None, change=True, lc=None, tf=None, tol=None, ncols=14):
    n = int(np.prod(case["np"]))
    lc = case["lc"] if lc is None else lc
    tf = case["tf"] if tf is None else tf
    mp = case["mp"] if mp is None else mp
    nsteps = int(round((tf - case["ti"]) / case["dt"])) + 4
    mxdct = max(n, nsteps // lc + 4)
    lnzvc = np.zeros((mxdct, ncols), order="F")
    u = np.array(case["psi"], dtype=np.float64)
    v = np.zeros(n)
    dim = {1: ".1D", 2: ".2D", 3: ".3D"}[len(case["np"])]
    absorb = case["absorb"] != 0
    info, mp_out = F.plnz(absorb=absorb, change=change, dim=dim, prtcrl=prtcrl,
                          tpabsor=TPABSOR[case["meta"].get("absorb")], lc=lc, lmtreort=10,
                          mp=mp, mpi=mp + 2, mpr=mp + 1, mxdct=mxdct, n=n, dt=case["dt"],
                          ti=case["ti"], tf=tf, tol=case["tol"] if tol is None else tol,
                          np_=case["np"], shm=case["shm"], vpot=case["vpot"], vabc=case["vabc"],
                          u=u, v=v, lnzvc=lnzvc)
    return dict(info=info, mp=mp_out, u=u, v=v, lnzvc=lnzvc, mpr=mp + 1, mpi=mp + 2)


@pytest.mark.parametrize("name", ["morse1d_sil", "morse1d_sil_smooth", "morse2d_sil"])
def test_plnz_matches_oracle_and_executable(oracle, capfd, name):
    case = G.setup_case(name)
    capfd.readouterr()
    got = call_plnz(case, ".PARTIAL")
    out, err = capfd.readouterr()
    assert err == ""
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_PARTIAL)
    nc, col = ref["nc"], got["lnzvc"]
    assert np.max(np.abs(col[:nc, got["mpr"] - 1] - ref["c"].real)) <= 1e-10
    assert np.max(np.abs(col[:nc, got["mpi"] - 1] - ref["c"].imag)) <= 1e-10
    assert np.max(np.abs(got["u"] - ref["u"])) <= 1e-10
    assert np.max(np.abs(got["v"] - ref["v"])) <= 1e-10
    assert got["info"] == ref["info"] and got["mp"] == 10
    # LNZVC(:, 1:MP) holds the last step's Lanczos basis (imaginary-part chain)
    n = got["u"].size
    basis = col[:n, :10]
    assert np.max(np.abs(basis.T @ basis - np.eye(10))) <= 1e-9
    assert not col[n:, :10].any()
    lines = out.split("\n")
    i = lines.index(" Partial auto-correlation function:")
    assert lines[i + 3] == ("          *t*       *Energy*        *Cr(t)*       *Ci(t)*    "
                            "*|C(t)|^2*      *|C|*")
    rows = np.array([[float(x) for x in l.split()] for l in lines[i + 4:] if len(l.split()) == 6])
    assert rows.shape == ref["rows"].shape
    e_ulp = 10.0 ** (np.floor(np.log10(np.abs(ref["rows"][:, 1]))) - 5)
    d = np.abs(rows - ref["rows"])
    assert np.all(d[:, [0, 2, 3, 4, 5]] <= np.array([5e-9, 5e-8, 5e-8, 5e-9, 5e-7]) + 1e-10)
    assert np.all(d[:, 1] <= 0.5 * e_ulp * 1.001)
    gold = case["data"]["rows"]
    dg = np.abs(rows - gold)
    assert np.all(dg[:, [0, 2, 3, 4, 5]] <= np.array([1e-8, 2e-7, 2e-7, 4e-7, 1e-6]) * 1.01)


@pytest.mark.parametrize("change", [True, False])
def test_plnz_order_messages_match_executable(capfd, change):
    """MP = 12 > LMTREORT = 10: LNZ's messages between the rows, MP lowered
    with *CHANGE (the executable's text, tests/golden/morse1d_sil_mp12_*.txt)."""
    case = G.setup_case("morse1d_sil")
    tf = 8 * case["dt"]
    capfd.readouterr()
    got = call_plnz(case, ".PARTIAL", mp=12, change=change, lc=2, tf=tf)
    out, err = capfd.readouterr()
    assert err == "" and got["info"] == 0
    assert got["mp"] == (10 if change else 12)
    name = "morse1d_sil_mp12_" + ("change" if change else "nochange")
    with open(f"{G.GOLDEN}/{name}.txt") as f:
        want = f.read().split("\n")[:-1]
    have = out.split("\n")[:-1]
    assert len(have) == len(want)
    for h, w in zip(have, want):
        if len(w.split()) == 6 and w.split()[0][0].isdigit():
            hv, wv = np.array(h.split(), float), np.array(w.split(), float)
            assert np.all(np.abs(hv - wv) <= np.array([1e-8, 1e-6 * abs(wv[1]), 1.01e-7,
                                                       1.01e-7, 1.01e-8, 1.01e-6])), (h, w)
        else:
            assert h == w


def test_pspofft_2d_golden_deck(oracle, capfd):
    """PSPOFFT with DIM = '.2D' on the 32x32 coupled-Morse golden deck: the
    reference's 2D kinetic table and in-place multiply, LNZVC, psi, TC and the
    printed rows against the oracle and the executable."""
    case = G.setup_case("morse2d_spo")
    capfd.readouterr()
    n = int(np.prod(case["np"]))
    nsteps = 2 * int(round((case["tf"] - case["ti"]) / case["dt"])) + 4
    lnzvc = np.zeros((nsteps + 4, 4), order="F")
    u1, v1, tc = np.array(case["psi"], dtype=np.float64), np.zeros(n), np.zeros(n)
    info = F.pspofft(absorb=False, dim=".2D", prtcrl=".PARTIAL", tpabsor=".NONE", lc=case["lc"],
                     mpi=3, mpr=2, mxdct=nsteps + 4, n=n, dt=case["dt"], ti=case["ti"],
                     tf=case["tf"], tol=case["tol"], np_=case["np"], sh=case["sh"], sm=case["sm"],
                     u1=u1, v1=v1, tc=tc, vpot=case["vpot"], vabc=None, lnzvc=lnzvc)
    out, err = capfd.readouterr()
    assert err == ""
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_PARTIAL)
    assert info == ref["info"]
    nc = ref["nc"]
    assert np.max(np.abs(lnzvc[:nc, 1] - ref["c"].real)) <= 1e-10
    assert np.max(np.abs(lnzvc[:nc, 2] - ref["c"].imag)) <= 1e-10
    assert np.max(np.abs(u1 - ref["u"])) <= 1e-10 and np.max(np.abs(v1 - ref["v"])) <= 1e-10
    npa = np.array(case["np"] + [1], dtype=np.int32)
    import ctypes as C
    tref, bb = np.zeros(n), C.c_double()
    oracle.lib().orc_digt(2, oracle._ip(npa), oracle._p(oracle.f64(case["sh"] + [1.0])),
                          oracle._p(oracle.f64(case["sm"] + [1.0])), oracle._p(tref),
                          C.byref(bb), case["ref_quirks"])
    assert np.array_equal(tc, tref)
    rows, _ = parse_table(out)
    assert rows.shape == ref["rows"].shape
    e_ulp = 10.0 ** (np.floor(np.log10(np.abs(ref["rows"][:, 1]))) - 5)
    d = np.abs(rows - ref["rows"])
    assert np.all(d[:, [0, 2, 3, 4, 5]] <= np.array([5e-9, 5e-8, 5e-8, 5e-9, 5e-7]) + 1e-10)
    assert np.all(d[:, 1] <= 0.5 * e_ulp * 1.001)
    gold = case["data"]["rows"]
    dg = np.abs(rows - gold)
    assert np.max(dg[:, [2, 3]]) <= 4e-6  # the oracle's pin to the executable on this deck


def test_psodfft_2d_golden_deck(oracle, capfd):
    """PSODFFT with DIM = '.2D' on the 32x32 coupled-Morse golden deck: the
    reference's 2D kinetic table makes this deck overflow within a few steps
    (the executable prints NaN from step 2 on); LNZVC follows the oracle
    relative to the magnitude until the overflow, psi(TF) and psi(TF - dt)
    have overflowed on both, TC equals the oracle's, and C(t) the finite
    values the executable printed."""
    from test_gpu_spond import close_until_overflow

    case = G.setup_case("morse2d_sod")
    capfd.readouterr()
    n = int(np.prod(case["np"]))
    nsteps = 2 * int(round((case["tf"] - case["ti"]) / case["dt"])) + 4
    lnzvc = np.zeros((nsteps + 4, 4), order="F")
    u1, v1, tc = np.array(case["psi"], dtype=np.float64), np.zeros(n), np.zeros(n)
    u2, v2 = np.zeros(n), np.zeros(n)
    info = F.psodfft(absorb=False, dim=".2D", prtcrl=".PARTIAL", tpabsor=".NONE", lc=case["lc"],
                     mpi=3, mpr=2, mxdct=nsteps + 4, n=n, dt=case["dt"], ti=case["ti"],
                     tf=case["tf"], tol=case["tol"], np_=case["np"], sh=case["sh"], sm=case["sm"],
                     u1=u1, v1=v1, u2=u2, v2=v2, tc=tc, vpot=case["vpot"], vabc=None,
                     lnzvc=lnzvc)
    capfd.readouterr()
    ref = G.run_oracle(case, case["ref_quirks"], prtcrl=oracle.PRT_PARTIAL)
    assert info == ref["info"]
    nc = ref["nc"]
    close_until_overflow(lnzvc[:nc, 1] + 1j * lnzvc[:nc, 2], ref["c"])
    for got, r in ((u2 + 1j * v2, ref["u"] + 1j * ref["v"]),
                   (u1 + 1j * v1, ref["u_prev"] + 1j * ref["v_prev"])):
        assert not np.isfinite(r).any() and not np.isfinite(got).any()
    npa = np.array(case["np"] + [1], dtype=np.int32)
    import ctypes as C
    tref, bb = np.zeros(n), C.c_double()
    oracle.lib().orc_digt(2, oracle._ip(npa), oracle._p(oracle.f64(case["sh"] + [1.0])),
                          oracle._p(oracle.f64(case["sm"] + [1.0])), oracle._p(tref),
                          C.byref(bb), case["ref_quirks"])
    assert np.array_equal(tc, tref)
    gold = case["data"]["rows"]
    ok = np.isfinite(gold[:, 2])
    rel = np.abs(lnzvc[:nc, 1][ok] - gold[ok, 2]) / np.maximum(1.0, np.abs(gold[ok, 2]))
    assert rel.max() < 1e-6


# ---------------------------------------------------------------------------
def call_psod(case, prtcrl, lc=None, tf=None, tol=None, ncols=4, mpr=2, mpi=3, psi=None):
    n = int(np.prod(case["np"]))
    lc = case["lc"] if lc is None else lc
    tf = case["tf"] if tf is None else tf
    nsteps = int(round((tf - case["ti"]) / case["dt"])) + 4
    mxdct = nsteps // lc + 4
    lnzvc = np.zeros((mxdct, ncols), order="F")
    psi = np.asarray(case["psi"] if psi is None else psi)
    u1, v1 = np.array(psi.real, dtype=np.float64), np.array(np.imag(psi), dtype=np.float64)
    u2, v2 = np.zeros(n), np.zeros(n)
    dim = {1: ".1D", 2: ".2D", 3: ".3D"}[len(case["np"])]
    info = F.psod(absorb=case["absorb"] != 0, dim=dim, prtcrl=prtcrl,
                  tpabsor=TPABSOR[case["meta"].get("absorb")], lc=lc, mpi=mpi, mpr=mpr,
                  mxdct=mxdct, n=n, dt=case["dt"], ti=case["ti"], tf=tf,
                  tol=case["tol"] if tol is None else tol, np_=case["np"], shm=case["shm"],
                  vpot=case["vpot"], vabc=case["vabc"], u1=u1, v1=v1, u2=u2, v2=v2, lnzvc=lnzvc)
    return dict(info=info, u=u2, v=v2, u_prev=u1, v_prev=v1, lnzvc=lnzvc)


def psod_oracle(oracle, case, prtcrl, lc=None, tf=None, tol=None, psi=None):
    p = oracle.make_prop(case["np"], case["dt"], case["ti"], case["tf"] if tf is None else tf,
                         case["sh"], case["sm"], lc=case["lc"] if lc is None else lc,
                         tol=case["tol"] if tol is None else tol, absorb=case["absorb"],
                         prtcrl=prtcrl, quirks=case["ref_quirks"], shm=case["shm"])
    psi = np.asarray(case["psi"] if psi is None else psi)
    return oracle.psod(p, case["vpot"], psi.real, np.imag(psi), vabc=case["vabc"])


@pytest.mark.parametrize("name", ["morse1d_psod", "morse1d_psod_voptic", "morse1d_psod_smooth",
                                  "morse2d_psod"])
def test_psod_dropin_matches_oracle_and_executable(oracle, capfd, name):
    case = G.setup_case(name)
    capfd.readouterr()
    got = call_psod(case, ".PARTIAL")
    out, err = capfd.readouterr()
    assert err == ""
    ref = psod_oracle(oracle, case, oracle.PRT_PARTIAL)
    nc, col = ref["nc"], got["lnzvc"]
    assert np.max(np.abs(col[:nc, 1] - ref["c"].real)) <= 1e-10
    assert np.max(np.abs(col[:nc, 2] - ref["c"].imag)) <= 1e-10
    assert not np.any(col[nc:, 1:3]) and not np.any(col[:, [0, 3]])
    for k in ("u", "v", "u_prev", "v_prev"):
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-10, k
    assert got["info"] == ref["info"]
    lines = out.split("\n")
    i = lines.index(" Partial auto-correlation function:")
    assert lines[i + 3] == ("       *t/fs*       *E/a.u.*        *Cr(t)*       *Ci(t)*    "
                            "*|C(t)|^2*      *|C|*")
    text = [l for l in lines[i + 4:] if len(l.split()) == 6]
    rows = np.array([[float(x) for x in l.split()] for l in text])
    assert rows.shape == ref["rows"].shape
    e_ulp = 10.0 ** (np.floor(np.log10(np.abs(ref["rows"][:, 1]))) - 5)
    d = np.abs(rows - ref["rows"])
    assert np.all(d[:, [0, 2, 3, 4, 5]] <= np.array([5e-9, 5e-8, 5e-8, 5e-9, 5e-7]) + 1e-10)
    assert np.all(d[:, 1] <= 0.5 * e_ulp * 1.001)
    gold = case["data"]["rows"]
    dg = np.abs(rows - gold)
    assert np.all(dg[:, [0, 2, 3, 4, 5]] <= np.array([1e-8, 1e-7, 1e-7, 1e-8, 1e-6]) * 1.01)
    assert np.all(dg[:, 1] <= e_ulp * 1.01)
    if name == "morse1d_psod":
        with open(f"{G.GOLDEN}/{name}_partial.txt") as f:
            want = f.read().split("\n")
        assert lines[i - 1:i + 4] == want[:5]
        same = sum(a == b for a, b in zip(text[:150], want[5:5 + 150]))
        assert same >= 140, same


def test_psod_dropin_complex_state_stride_and_info(oracle, capfd):
    """A complex initial state (the restart-copy defect of psod.f:136-141 acts
    on V), LC = 5 into columns 5/6 without printing, and INFO on four
    tolerances (the norm column squared in the loop, psod.f:183)."""
    case = G.setup_case("morse1d_psod")
    n = len(case["psi"])
    psi = case["psi"] * np.exp(0.7j * np.sin(np.arange(n) / 37.0))
    tf = 150 * case["dt"]
    capfd.readouterr()
    got = call_psod(case, ".NO", lc=5, tf=tf, ncols=8, mpr=5, mpi=6, psi=psi)
    assert capfd.readouterr().out == ""
    ref = psod_oracle(oracle, case, oracle.PRT_NONE, lc=5, tf=tf, psi=psi)
    nc, col = ref["nc"], got["lnzvc"]
    assert np.max(np.abs(col[:nc, 4] + 1j * col[:nc, 5] - ref["c"])) <= 1e-10
    for k in ("u", "v", "u_prev", "v_prev"):
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-10, k
    for tol in (1e-12, 1e-7, 1e-3, 10.0):
        got = call_psod(case, ".YES", tol=tol, tf=tf, psi=psi)
        ref = psod_oracle(oracle, case, oracle.PRT_YES, tol=tol, tf=tf, psi=psi)
        assert got["info"] == ref["info"], (tol, got["info"], ref["info"])
    capfd.readouterr()
