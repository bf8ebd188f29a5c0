#!/usr/bin/env python3
"""Generate the golden fixtures that pin the CPU oracle to eSPec itself.

Run where the reference tree is available (its path in the ESPEC_REF
environment variable, or the default below).  The script only RUNS the shipped
eSPec executable (espec_v07.x) as a black box on input decks, and reads the
reference's own test fixtures (ttests/) as text; it never inspects the
executable.  Outputs go to tests/golden/*.npz plus manifest.json.

Cases:
  test8       reference test 8 (.ONLYSPEC): C(t) from ttests/correl8.inp ->
              HWHM -> SPECTRUMTD, compared with the executable's spectrum and
              with ttests/results.test8 (the reference's committed golden).
  test4       reference test 4 (.PSIL, N=201 from ttests/eigpot_test3.inp):
              partial C(t) table and spectrum from the executable.
  morse1d_*   1D Morse (N=1024 on [0.5, 8.0] bohr, mass 918 m_e, Gaussian at
              1.8 bohr, sigma 0.2) at dt = 0.005 au for 2048 steps with .PFSOD,
              .PFSPO and .PSIL, without absorber, with a .VOPTIC_POLIN CAP and
              with a .SMOOTHW mask.
  morse2d_*   2D coupled Morse on a 32x32 grid with .PSIL, .PFSPO and .PFSOD
              (the last two pin the reference's 2D kinetic-table defect).
  *_psod*     the same 1D decks and the 2D deck with .PSOD (second-order
              differences with the finite-difference Hamiltonian).  With
              --psod-only only these are generated and merged into the
              manifest.
  deck_*      whole decks for the deck driver (input.spc, wf_pot.inp and the
              executable's output from the propagation on); --decks-only
              [name ...] generates only these (or the named ones).
  calc2d_*    2D decks with computed initial states (.CALC, .MTRXDIAG) and the
              executable's output, with its MAKECST lines (constants.txt);
              --calc2d-only generates only these.
  makecst_lines.json  MAKECST's printed constants for every named 1D/2D form
              (a .PES deck each); --makecst-only generates only these.
  collision_* a Gaussian wave packet with momentum (.COLLISION) in a 1D well,
              .PSOD and .PFSPO; --collision-only generates only these.
  ti_*        the time-independent formalism (.ENERGY, .SPECTRUM .TI) on the
              surfaces of reference test 12 and of calc2d_ohs_psil; the
              executable's output from its first "Calculating eigenvalue(s)"
              line; --ti-only generates only these.
  reftest*    the reference's own test decks ttests/input.test<i> (most with
              an analytic potential and a computed initial state, .CALC):
              the deck as input.spc and the executable's output from the
              propagation on, gzipped, as expected.txt.gz; --reftests-only
              [i ...] generates only these.  Tests 1 and 5 are left out: the
              executable stops in their .LANCZS diagonalisation (DSTEIN is
              called with an illegal argument); tests 2 and 3 run edited (REFTEST_EDITS).
"""
import gzip
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

REF = os.environ.get("ESPEC_REF", "/root/reference")
BIN = os.path.join(REF, "espec_v07.x")
OUT = os.path.dirname(os.path.abspath(__file__))

SHFS = 2.4188843243e-2
AMU = 1836.152667539


def run_deck(deck, files, timeout=600):
    d = tempfile.mkdtemp(prefix="espec_golden_")
    try:
        with open(os.path.join(d, "input.spc"), "w") as f:
            f.write(deck)
        for name, src in files.items():
            dst = os.path.join(d, name)
            if isinstance(src, str) and os.path.exists(src):
                os.symlink(src, dst)
            else:
                with open(dst, "w") as f:
                    f.write(src)
        r = subprocess.run([BIN], cwd=d, capture_output=True, timeout=timeout)
        return r.stdout.decode("utf-8", errors="replace")
    finally:
        shutil.rmtree(d, ignore_errors=True)


def _floats(line):
    # Fortran prints '****' when a value overflows its edit descriptor
    return [np.nan if "*" in x else float(x.replace("D", "E")) for x in line.split()]


def parse_partial(out):
    lines = out.splitlines()
    for i, l in enumerate(lines):
        if "Partial auto-correlation function:" in l:
            break
    else:
        raise RuntimeError("no partial correlation table:\n" + out[-3000:])
    rows = []
    for l in lines[i + 4:]:
        s = l.split()
        if len(s) != 6:
            if rows:
                break
            continue
        try:
            rows.append(_floats(l))
        except ValueError:
            rows.append([np.nan] * 6)
    return np.array(rows)


def parse_table(out, header, ncol):
    lines = out.splitlines()
    for i, l in enumerate(lines):
        if l.strip() in (header if isinstance(header, tuple) else (header,)):
            break
    else:
        raise RuntimeError("no table " + header)
    rows = []
    for l in lines[i + 1:]:
        s = l.split()
        if len(s) == ncol:
            try:
                rows.append(_floats(l))
                continue
            except ValueError:
                pass
        if rows:
            break
    return np.array(rows)


def partial_text(out, first=150, last=50):
    """The head of the partial auto-correlation table as printed (the lines
    from the blank line before its title to the column titles) and the text
    of its first and last rows, for pinning the drop-ins' Fortran output."""
    lines = out.splitlines()
    for i, l in enumerate(lines):
        if "Partial auto-correlation function:" in l:
            break
    head = lines[i - 1:i + 4]
    rows = []
    for l in lines[i + 4:]:
        if len(l.split()) != 6:
            break
        rows.append(l)
    keep = rows[:first] + rows[-last:]
    return "\n".join(head + keep) + "\n", len(rows)


TEXT_CASES = ("morse1d_spo", "morse1d_sod", "morse1d_spo_voptic", "morse1d_psod")


def case_test8_text():
    """Reference test 8 run by the executable: the printed spectrum block
    (SPECTRUMTD, spectrumtd.f:83-98) -- its head, first 100 and last 20 rows."""
    tt = os.path.join(REF, "ttests")
    deck = open(os.path.join(tt, "input.test8")).read()
    out = run_deck(deck, {"correl8.inp": os.path.join(tt, "correl8.inp")})
    lines = out.splitlines()
    i = [k for k, l in enumerate(lines) if l.strip() == "Spectrum:"][0]
    rows = []
    for l in lines[i + 3:]:
        if len(l.split()) != 4:
            break
        rows.append(l)
    with open(os.path.join(OUT, "test8_spectrum.txt"), "w") as f:
        f.write("\n".join(lines[i - 1:i + 3] + rows[:100] + rows[-20:]) + "\n")


def case_sil_order_text(change):
    """.PSIL with MP = 12 > LMTREORT = 10 (param.f:9) for 8 steps (LC = 2): the
    printed block from the table head to the end of propagation, with LNZ's
    order messages (lnz.f:64-72) between the rows, *CHANGE .YES or .NO."""
    x, psi, v = morse1d_inputs()
    dt_fs = 0.005 * SHFS
    deck = DECK.format(title="sil order", dim=".1D", np="1024", mass=fmt(918.0 / AMU),
                       prop=".PSIL", tf=fmt(8 * dt_fs), dt=fmt(dt_fs), mp="  12", absorb="",
                       mf=3)
    deck = deck.replace("*CHANGE\n.YES", "*CHANGE\n" + change)
    out = run_deck(deck, {"wf_pot.inp": write_1d_file(x, psi, v)})
    lines = out.splitlines()
    i = [k for k, l in enumerate(lines) if "Partial auto-correlation function:" in l][0]
    j = [k for k, l in enumerate(lines) if "Eigenvector propagated." in l][0]
    name = "morse1d_sil_mp12_" + ("change" if change == ".YES" else "nochange")
    with open(os.path.join(OUT, name + ".txt"), "w") as f:
        f.write("\n".join(lines[i - 1:j]) + "\n")


def fmt(x):
    return repr(float(x))


def write_1d_file(x, psi, v):
    s = ["# Eigenvector:"]
    s += [f" {fmt(a)}   {fmt(b)}" for a, b in zip(x, psi)]
    s += ["# Final potential values:"]
    s += [f" {fmt(a)}   {fmt(b)}" for a, b in zip(x, v)]
    return "\n".join(s) + "\n"


def write_2d_file(x, y, psi, v):
    # rows "y x value" with x fastest (rdpte.f reads (XI(I), I=ND,1,-1), V)
    s = ["# Eigenvector:"]
    for j, yy in enumerate(y):
        for i, xx in enumerate(x):
            s.append(f" {fmt(yy)}  {fmt(xx)}   {fmt(psi[j, i])}")
    s.append("# Final potential values:")
    for j, yy in enumerate(y):
        for i, xx in enumerate(x):
            s.append(f" {fmt(yy)}  {fmt(xx)}   {fmt(v[j, i])}")
    return "\n".join(s) + "\n"


DECK = """*** eSPec input file ***
========================
**MAIN
*TITLE
 golden fixture {title}
*DIMENSION
{dim}
 {np}/
*POTENTIAL
.FILE
wf_pot.inp
*MASS
 {mass}/
*TPCALC
.SPECTRUM
.TD
*INIEIGVC
.GETR
*CHANGE
.YES
*SHIFT_POTENTIAL
.NO
*PRTCRL
.PARTIAL

**TD
*PROPAG
{prop}
 0.0  {tf}  {dt}{mp}/
*PRPGSTATE
 0/
*TPTRANS
.ONE
*PRPTOL
 1D3/
{absorb}
**SPECTRUM
*FOURIER
 {mf}/
*WINDOWING
.SG
 1D-3/
**END
"""


def morse1d_inputs():
    n = 1024
    x = 0.5 + np.arange(n) * (7.5 / 1023)
    v = 0.17 * (1 - np.exp(-1.0 * (x - 1.4))) ** 2
    psi = np.exp(-((x - 1.8) ** 2) / (2 * 0.2 ** 2))
    psi = psi / np.sqrt(np.sum(psi ** 2))
    # round-trip through the text the executable reads
    x = np.array([float(fmt(a)) for a in x])
    v = np.array([float(fmt(a)) for a in v])
    psi = np.array([float(fmt(a)) for a in psi])
    return x, psi, v


def morse2d_inputs():
    nx, ny = 32, 32
    x = 1.0 + np.arange(nx) * (1.0 / (nx - 1))
    y = 1.2 + np.arange(ny) * (1.2 / (ny - 1))
    X, Y = np.meshgrid(x, y)  # [j, i]
    v = (0.17 * (1 - np.exp(-1.0 * (X - 1.4))) ** 2 + 0.12 * (1 - np.exp(-1.2 * (Y - 1.8))) ** 2
         + 0.01 * (X - 1.4) * (Y - 1.8))
    psi = np.exp(-((X - 1.5) ** 2) / (2 * 0.1 ** 2) - ((Y - 1.8) ** 2) / (2 * 0.12 ** 2))
    psi = psi / np.sqrt(np.sum(psi ** 2))
    r = lambda a: np.vectorize(lambda t: float(fmt(t)))(a)
    return r(x), r(y), r(psi), r(v)


def case_morse1d(name, prop, absorb_block, absorb_meta):
    x, psi, v = morse1d_inputs()
    dt_fs = 0.005 * SHFS
    nsteps = 2048
    tf = nsteps * dt_fs
    mass_amu = 918.0 / AMU
    mp = "  10" if prop == ".PSIL" else ""
    deck = DECK.format(title=name, dim=".1D", np="1024", mass=fmt(mass_amu), prop=prop,
                       tf=fmt(tf), dt=fmt(dt_fs), mp=mp, absorb=absorb_block, mf=12)
    out = run_deck(deck, {"wf_pot.inp": write_1d_file(x, psi, v)})
    if name in TEXT_CASES:
        text, nrows = partial_text(out)
        with open(os.path.join(OUT, name + "_partial.txt"), "w") as f:
            f.write(text)
    rows = parse_partial(out)
    corr = parse_table(out, "*t/fs*       *C(t)r*       *C(t)i*", 3)
    spec = parse_table(out, "*E (eV)*           *W*           *FFTr*          *FFTi*", 4)
    meta = dict(kind="morse1d", prop=prop, np=[1024], dt_fs=dt_fs, tf_fs=tf, mass_amu=mass_amu,
                mp=10, mf=12, window="SG", wp=1e-3, **absorb_meta)
    # x, psi, v are regenerated by morse1d_inputs(); the energy axis of the
    # spectrum overflows its F12.7 field at this dt, so only C(t) is kept.
    arrays = dict(rows=rows)
    if name in ("morse1d_sod", "morse1d_spo_voptic"):
        # total C(t) table (espec.f:1545-1576).  Not kept for .PSIL: there the
        # reference stores C(t) past the end of its LNZVC array and the table
        # is corrupted before it is printed.
        arrays["corr"] = corr
    if name == "morse1d_sod":
        arrays.update(x=x, psi=psi, v=v)
    return meta, arrays


def case_morse2d(name, prop):
    x, y, psi, v = morse2d_inputs()
    dt_fs = 0.005 * SHFS
    nsteps = 512
    tf = nsteps * dt_fs
    m1, m2 = 918.0 / AMU, 1500.0 / AMU
    mp = "  10" if prop == ".PSIL" else ""
    deck = DECK.format(title=name, dim=".2D", np="32 32", mass=f"{fmt(m1)} {fmt(m2)}", prop=prop,
                       tf=fmt(tf), dt=fmt(dt_fs), mp=mp, absorb="", mf=10)
    out = run_deck(deck, {"wf_pot.inp": write_2d_file(x, y, psi, v)})
    rows = parse_partial(out)
    meta = dict(kind="morse2d", prop=prop, np=[32, 32], dt_fs=dt_fs, tf_fs=tf,
                mass_amu=[m1, m2], mp=10, mf=10)
    return meta, dict(x=x, y=y, psi=psi, v=v, rows=rows)


def case_test4():
    tt = os.path.join(REF, "ttests")
    deck = open(os.path.join(tt, "input.test4")).read()
    out = run_deck(deck, {"eigpot_test3.inp": os.path.join(tt, "eigpot_test3.inp")})
    rows = parse_partial(out)
    lines = open(os.path.join(tt, "eigpot_test3.inp")).read().splitlines()
    data = [_floats(l) for l in lines if l.strip() and not l.startswith("#")]
    data = np.array(data)
    x, psi, v = data[:201, 0], data[:201, 1], data[201:402, 1]
    golden_v04 = parse_partial(open(os.path.join(tt, "results.test4")).read())
    meta = dict(kind="test4", prop=".PSIL", np=[201], mass_amu=7.49, ti_fs=0.0, tf_fs=250.0,
                dt_fs=2e-3, mp=10, change=True, mf=12, hwhm=[0.087, 0.0, 0.12, 19.562],
                shiftp=True, tol=3.0)
    # the total C(t) and spectrum of this run are not kept: the reference
    # stores C(t) past the end of its LNZVC array (MP+1 > LMTREORT) and the
    # .PSIL path overwrites some of those samples before they are assembled
    return meta, dict(x=x, psi=psi, v=v, rows=rows, rows_v04=golden_v04)


def case_test8():
    tt = os.path.join(REF, "ttests")
    deck = open(os.path.join(tt, "input.test8")).read()
    out = run_deck(deck, {"correl8.inp": os.path.join(tt, "correl8.inp")})
    spec = parse_table(out, "*E (eV)*           *W*           *FFTr*          *FFTi*", 4)
    cin = parse_table(open(os.path.join(tt, "correl8.inp")).read(),
                      "*t/fs*       *C(t)r*       *C(t)i*", 3)
    gold = parse_table(open(os.path.join(tt, "results.test8")).read(),
                       ("*E/eV*           *W*           *FFTr*          *FFTi*",), 4)
    meta = dict(kind="test8", mf=13, hwhm=[0.08, 0.0, 0.0, 0.0], window="NONE",
                executable_equals_committed_golden=bool(np.array_equal(spec, gold)))
    arrays = dict(cin=cin, spec_golden=gold)
    if not np.array_equal(spec, gold):
        arrays["spec"] = spec
    return meta, arrays


VOPTIC = """*ABSORBING
.VOPTIC_POLIN
 -0.02  2.0  0.0/
 1.6  2.2  0.0 0.0 0.0 0.0/
"""
SMOOTH = """*ABSORBING
.SMOOTHW
 0.05  1.0  0.0/
 1.55  2.3  0.0 0.0 0.0 0.0/
"""


PULSE_EXP = """*PULSE_AND_DIPOLE
.GAUS
 5.0D7  0.1  2.5  0.15  0.0/
.EXP
 0.5 0.3 0.0/
"""
PULSE_GGAUS_CONST = """*PULSE_AND_DIPOLE
.GGAUS
 3.0D11  0.1  2.5  0.15  0.3  4.0/
.CONST
 0.8/
"""
PULSE_SIN2_EXP = """*PULSE_AND_DIPOLE
.SIN2
 5.0D7  0.2  2.5  0.05  0.0/
.EXP
 0.5 0.3 0.0/
"""
VOPTIC_SMALL = """*ABSORBING
.VOPTIC_POLIN
 -0.5  2.0  0.0/
 0.9  6.5  0.0 0.0 0.0 0.0/
"""
SMOOTH_SMALL = """*ABSORBING
.SMOOTHW
 0.05  1.0  0.0/
 0.9  6.5  0.0 0.0 0.0 0.0/
"""


DECK_CASES = {
    # name: (dimension, propagator, MP field, absorber block, HWHM block)
    "deck_spo_hwhm": (1, ".PFSPO", "", "", "*HWHM\n 0.05 0.0 0.0 0.0/\n"),
    "deck_psod_voptic": (1, ".PSOD", "", VOPTIC_SMALL, ""),
    "deck_sil_smooth": (1, ".PSIL", "  10", SMOOTH_SMALL, ""),
    "deck_sil_2d": (2, ".PSIL", "  10", "", ""),
    "deck_ppsod": (1, ".PPSOD", "", PULSE_EXP, ""),
    # NPR = 2, KP = 0 becomes NPR = 1 (rdinput.f:659): |<W1|psi>|^2 with W1 the
    # deck's own eigenvector, LNZVC(., KP+1) = EIGVC(., 1)
    "deck_ppsod_proj": (1, ".PPSOD", "", PULSE_EXP + "*NPROJECTIONS\n 2 0/\n", ""),
    "deck_ppsil": (1, ".PPSIL", "  10", PULSE_EXP, ""),
    # NPR = 3, KP = 0 becomes NPR = 2: PPLNZ prints |C|^2 and |<W1|psi>|^2
    "deck_ppsil_proj": (1, ".PPSIL", "  10", PULSE_EXP + "*NPROJECTIONS\n 3 0/\n", ""),
    # 2D: DIPLMMT's R = XI(1) + (I - 1) SH(1) runs over all NT points of the grid
    "deck_ppsod_2d": (2, ".PPSOD", "", PULSE_EXP, ""),
    "deck_ppsil_2d": (2, ".PPSIL", "  10", PULSE_EXP, ""),
    # the other pulse shapes of ef.f and the .CONST dipole (mu = c / R)
    "deck_ppsod_ggaus": (1, ".PPSOD", "", PULSE_GGAUS_CONST, ""),
    "deck_ppsod_sin2": (1, ".PPSOD", "", PULSE_SIN2_EXP, ""),
}


def case_deck(name):
    """A whole deck for the deck driver: input.spc and wf_pot.inp under
    tests/golden/<name>/, and the executable's output from its last
    'Propagating eigenvector...' line to the end as expected.txt.  Small grids
    (N = 256 on [0.5, 8] bohr, or the 32 x 32 2D grid), 256 steps, MF = 8."""
    nd, prop, mp, absorb, hwhm = DECK_CASES[name]
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    if nd == 1:
        n = 256
        x = 0.5 + np.arange(n) * (7.5 / (n - 1))
        v = 0.17 * (1 - np.exp(-1.0 * (x - 1.4))) ** 2
        psi = np.exp(-((x - 1.8) ** 2) / (2 * 0.2 ** 2))
        psi = psi / np.sqrt(np.sum(psi ** 2))
        wf = write_1d_file(x, psi, v)
        dim, npt, mass = ".1D", "256", fmt(918.0 / AMU)
        dt_fs = 0.05 * SHFS
    else:
        x, y, psi, v = morse2d_inputs()
        wf = write_2d_file(x, y, psi, v)
        dim, npt, mass = ".2D", "32 32", f"{fmt(918.0 / AMU)} {fmt(1500.0 / AMU)}"
        dt_fs = 0.005 * SHFS
    deck = DECK.format(title=name, dim=dim, np=npt, mass=mass, prop=prop, tf=fmt(256 * dt_fs),
                       dt=fmt(dt_fs), mp=mp, absorb=absorb, mf=8)
    if hwhm:
        deck = deck.replace("**SPECTRUM\n*FOURIER", "**SPECTRUM\n" + hwhm + "*FOURIER")
    if prop in (".PPSOD", ".PPSIL"):  # propagation only; the pulse block goes to **TD
        deck = deck.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.PROPAGATION")
    with open(os.path.join(d, "input.spc"), "w") as f:
        f.write(deck)
    with open(os.path.join(d, "wf_pot.inp"), "w") as f:
        f.write(wf)
    out = run_deck(deck, {"wf_pot.inp": wf})
    lines = out.splitlines()
    i = max(k for k, l in enumerate(lines) if l.strip() == "Propagating eigenvector...")
    with open(os.path.join(d, "expected.txt"), "w") as f:
        f.write("\n".join(lines[i - 1:]) + "\n")


# Edited decks.  Test 2 runs with .MTRXDIAG in place of its .LANCZS: on its
# 560-point grid the executable's LANCZS returns ghost eigenvalues (0.0132557
# and 0.0190582 twice each) and propagates a vector of norm^2 1.94 as "state
# 2".  Test 3 (.PPSOD with the dipole file dipol2.inp and populations of six
# computed states) runs 40 fs instead of 2000 with its .GGAUS pulse moved into
# that window (TP 10 fs, T0 20 fs), and with .MTRXDIAG: its LANCZS states above
# the ground state include a ghost as well (test 9's table: 0.0275652).
LANCZS_TO_MTRXDIAG = ("*TPDIAG\n.LANCZS", "*TPDIAG\n.MTRXDIAG")
REFTEST_EDITS = {
    "2_mtrxdiag": [LANCZS_TO_MTRXDIAG],
    "3_short": [LANCZS_TO_MTRXDIAG, (" 0.0  2000.0  5D-5  10/", " 0.0  40.0  5D-5  10/"),
                (" 1.5D+12  100.0  0.241  700.0  4.7124   1.0/",
                 " 1.5D+12  10.0  0.241  20.0  4.7124   1.0/")],
}
REFTEST_FILES = {"3_short": ["dipol2.inp"], "4": ["eigpot_test3.inp"]}
# test 8 (.ONLYSPEC) reads the correlation function of an old output file;
# its table (the lines from " Correlation Function:" on) is kept, gzipped
REFTEST_GZ_FILES = {"8": ["correl8.inp"]}
# test 4: .PSIL from the .FILE eigpot_test3.inp; test 15: .PES, the 2D
# .LEPS_CC potential (200 x 180 points) printed
REFTESTS = [6, 9, 10, 11, 12, 13, 14, "2_mtrxdiag", "3_short", 8, 4, 15]
MARKS = ("Propagating eigenvector...", "Getting correlation function...",
         "Generating initial potential...")


def case_reftest(i):
    """The reference's test deck i under tests/golden/reftest<i>/."""
    num = int(str(i).split("_")[0])
    with open(os.path.join(REF, "ttests", f"input.test{num}")) as f:
        deck = f.read()
    for old, new in REFTEST_EDITS.get(str(i), []):
        assert old in deck, (i, old)
        deck = deck.replace(old, new)
    d = os.path.join(OUT, f"reftest{i}")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.spc"), "w") as f:
        f.write(deck)
    files = {}
    for name in REFTEST_FILES.get(str(i), []):
        src = os.path.join(REF, "ttests", name)
        shutil.copyfile(src, os.path.join(d, name))
        files[name] = src
    for name in REFTEST_GZ_FILES.get(str(i), []):
        with open(os.path.join(REF, "ttests", name), "rb") as f:
            raw = f.read().decode("latin-1").split("\n")
        k = next(j for j, l in enumerate(raw) if l.startswith(" Correlation Function:"))
        text = "\n".join(raw[k:]) + "\n"
        with gzip.open(os.path.join(d, name + ".gz"), "wt") as f:
            f.write(text)
        files[name] = text
    out = run_deck(deck, files, timeout=3600)
    lines = out.splitlines()
    k = max(j for j, l in enumerate(lines) if l.strip() in MARKS)
    with gzip.open(os.path.join(d, "expected.txt.gz"), "wt") as f:
        f.write("\n".join(lines[k - 1:]) + "\n")


# 2D decks with computed initial states (.CALC with .MTRXDIAG on a 32 x 32
# grid): the harmonic .OHS surfaces in cm^-1 and angstrom, propagated on the
# final surface from its second state with .PSIL; and a .MORSE pair whose
# constants MAKECST leaves as written (it has no 2D .MORSE branch: the
# message, then the constants in atomic units), grid ranges in bohr
# ('*GRID_RANGES au'), with .PSOD.  (The executable's 2D .PFSPO diverges
# from the first step on such a deck: its 2D kinetic table fills TC(1..NP1)
# only.)
CALC2D = {
    "calc2d_ohs_psil": """*** eSPec input file ***
**MAIN
*TITLE
 2D harmonic surfaces, computed state 1, .PSIL
*DIMENSION
.2D
 32 32/
*POTENTIAL
.OHS
 1.14600  1943.79  1.14600  1700.00/
 1.21100  1629.23  1.18000  1800.00/
*GRID_RANGES
 0.85  1.45  0.90  1.50/
*MASS
 7.49D0  9.0D0/
*TPCALC
.SPECTRUM
.TD
*INIEIGVC
.CALC
*CHANGE
.YES
*PRTCRL
.PARTIAL
**TI
*TPDIAG
.MTRXDIAG
*NIST
 3  0/
**TD
*PROPAG
.PSIL
 0.0  4.0  2D-3  10/
*PRPGSTATE
 1/
*TPTRANS
.ONE
**SPECTRUM
*FOURIER
 8/
*WINDOWING
.SG
 1D-3/
**END
""",
    "calc2d_morse_psod": """*** eSPec input file ***
**MAIN
*TITLE
 2D Morse surfaces in atomic units, computed ground state, .PSOD
*DIMENSION
.2D
 32 32/
*POTENTIAL
.MORSE
 2.0  1.0  0.17  2.3  0.9  0.15/
 2.1  1.0  0.17  2.4  0.9  0.14/
*GRID_RANGES au
 1.45  2.65  1.75  2.95/
*MASS
 1.0D0  1.5D0/
*TPCALC
.SPECTRUM
.TD
*INIEIGVC
.CALC
*CHANGE
.YES
*PRTCRL
.PARTIAL
**TI
*TPDIAG
.MTRXDIAG
*NIST
 1  0/
**TD
*PROPAG
.PSOD
 0.0  5.0  2.5D-3/
*PRPGSTATE
 0/
*TPTRANS
.ONE
**SPECTRUM
*FOURIER
 9/
*WINDOWING
.SG
 1D-3/
**END
""",
}


# The time-independent formalism: eigenvalues only (.ENERGY) and the
# Franck-Condon spectrum of SPECTRUMTI (.SPECTRUM .TI) between the initial
# and final surfaces of reference test 12, and of the 2D .OHS deck above
def ti_decks():
    with open(os.path.join(REF, "ttests", "input.test12")) as f:
        t12 = f.read()
    energy = t12.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.ENERGY")
    ti = t12.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.SPECTRUM\n.TI")
    ti = ti.replace("*NIST\n 7  0/", "*NIST\n 2  0/\n*NFST\n 6  0/")
    ti2d = CALC2D["calc2d_ohs_psil"].replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.SPECTRUM\n.TI")
    ti2d = ti2d.replace("*NIST\n 3  0/", "*NIST\n 2  0/\n*NFST\n 5  0/")
    for d in (energy, ti, ti2d):
        assert d.count(".ENERGY") + d.count(".TI\n") == 1
    return {"ti_energy_ohs": energy, "ti_spectrum_ohs": ti, "ti_spectrum_2d_ohs": ti2d}


def case_ti(name, deck):
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.spc"), "w") as f:
        f.write(deck)
    out = run_deck(deck, {})
    lines = out.splitlines()
    k = min(j for j, l in enumerate(lines)
            if l.strip() == "Calculating eigenvalue(s) and eigenvector(s)")
    with open(os.path.join(d, "expected.txt"), "w") as f:
        f.write("\n".join(lines[k - 1:]) + "\n")


# .COLLISION: a Gaussian wave packet with momentum (init_cond.f) in a 1D
# harmonic well, propagated with .PSOD and with .PFSPO.  The complex initial
# state meets PSOD's restart copy (psod.f:136-141, V1(I+1) = V0(I)): its norm
# and energy drift until INFO = 1, and *DONOTSTOP lets the run end normally.
COLLISION = """*** eSPec input file ***
**MAIN
*TITLE
 a Gaussian wave packet with momentum in a harmonic well
*DIMENSION
.1D
 512/
*POTENTIAL
.OHS
 1.14600  1943.79/
 1.14600  1943.79/
*GRID_RANGES
 0.6  1.8/
*MASS
 7.49D0/
*TPCALC
.COLLISION
*INIEIGVC
.CALC
*CHANGE
.YES
*PRTCRL
.PARTIAL
*DONOTSTOP
.ON
**TI
*COLLISION_ENERGY
 0.05/
*INIT_POSSITION
 2.0/
*SIZE_OF_GAUSSIAN
 0.1/
**TD
*PROPAG
{prop}
**END
"""
COLLISION_DECKS = {"collision_psod": ".PSOD\n 0.0  20.0  2D-4/",
                   "collision_pfspo": ".PFSPO\n 0.0  20.0  2D-4/"}


def case_collision(name):
    deck = COLLISION.format(prop=COLLISION_DECKS[name])
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.spc"), "w") as f:
        f.write(deck)
    out = run_deck(deck, {})
    lines = out.splitlines()
    k = max(j for j, l in enumerate(lines) if l.strip() == "Propagating eigenvector...")
    with gzip.open(os.path.join(d, "expected.txt.gz"), "wt") as f:
        f.write("\n".join(lines[k - 1:]) + "\n")


# MAKECST's unit conversion (makecst.f:82-340) for every named form: a
# .PES deck per form with two constant records, and the lines the executable
# prints from " Initial potential:" to " Units converted."
MAKECST_FORMS = [
    (".1D", ".OHS", "1.146 1943.79", "1.211 1629.23"),
    (".1D", ".DOHS", "1.146 1943.79 1.2 1.3 1629.23", "1.211 1629.23 1.25 1.35 1500.0"),
    (".1D", ".MORSE", "1.146 1943.79 13.71", "1.211 1629.23 17.74"),
    (".1D", ".MORSE_CM^1", "1.146 1943.79 13.71", "1.211 1629.23 17.74"),
    (".1D", ".MORSE_Dalpha", "1.146 1.9 4.6", "1.211 2.1 3.1"),
    (".1D", ".MORSE_Dalpha_au", "2.17 1.0 0.17", "2.29 1.1 0.12"),
    (".1D", ".ANTI-MORSE", "1.146 1943.79 13.71", "1.211 1629.23 17.74"),
    (".1D", ".MORSEM", "1.146 1943.79 13.71", "1.211 1629.23 17.74"),
    (".1D", ".MOD-MORSE", "1.146 1943.79 13.71", "1.211 1629.23 17.74"),
    (".1D", ".BARRIER", "1.0 1.3 0.5", "1.1 1.4 0.6"),
    (".1D", ".BARRIER_au", "2.0 2.5 0.02", "2.1 2.6 0.03"),
    (".1D", ".CONST", "0.5", "0.7"),
    (".1D", ".FREE", "0.0", "0.0"),
    (".2D", ".OHS", "1.146 1943.79 1.146 1700.0", "1.211 1629.23 1.18 1800.0"),
    (".2D", ".LSM", "1.1 1.9 30000 2.1 25000 1.2 1.8 20000",
     "1.15 1.8 31000 2.0 24000 1.25 1.7 21000"),
    (".2D", ".LS", "1.1 1.9 30000 2.1 25000", "1.15 1.8 31000 2.0 24000"),
    (".2D", ".LEPS_Dalpha", "0.74 1.94 4.75 0.74 1.94 4.75 0.74 1.94 4.75 0.3 0.05 0.05 180",
     "0.74 1.94 4.75 0.74 1.94 4.75 0.74 1.94 4.75 0.3 0.05 0.05 180"),
    (".2D", ".BARRIERXY", "1.0 1.3 0.5 1.1 1.4 0.6", "1.0 1.3 0.5 1.1 1.4 0.6"),
    (".2D", ".WELLY", "1.0 1.3 0.5", "1.1 1.4 0.6"),
    (".2D", ".BARRIER", "1.0 1.3 1.1 1.4 0.5", "1.0 1.3 1.1 1.4 0.6"),
    (".2D", ".CONST", "0.5", "0.7"),
    (".2D", ".MORSE", "2.0 1.0 0.17 2.3 0.9 0.15", "2.1 1.0 0.17 2.4 0.9 0.14"),
]


def makecst_deck(dim, form, c1, c2):
    npt, ranges, mass = (" 64/", " 0.9  1.5/", " 7.49D0/") if dim == ".1D" else \
        (" 32 32/", " 0.9  1.5  0.9  1.5/", " 7.49D0  9.0D0/")
    return (f"*** eSPec input file ***\n**MAIN\n*TITLE\n MAKECST {form}\n*DIMENSION\n{dim}\n"
            f"{npt}\n*POTENTIAL\n{form}\n {c1}/\n {c2}/\n*GRID_RANGES\n{ranges}\n*MASS\n"
            f"{mass}\n*TPCALC\n.PES\n*INIEIGVC\n.CALC\n*CHANGE\n.YES\n**END\n")


def case_makecst():
    out = {}
    for dim, form, c1, c2 in MAKECST_FORMS:
        deck = makecst_deck(dim, form, c1, c2)
        lines = run_deck(deck, {}).splitlines()
        i = lines.index(" Initial potential:")
        j = lines.index(" Units converted.")
        out[f"{dim}{form}"] = {"deck": deck, "lines": lines[i:j - 1]}
    with open(os.path.join(OUT, "makecst_lines.json"), "w") as f:
        json.dump(out, f, indent=1)


def case_calc2d(name):
    deck = CALC2D[name]
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "input.spc"), "w") as f:
        f.write(deck)
    out = run_deck(deck, {})
    lines = out.splitlines()
    k = max(j for j, l in enumerate(lines) if l.strip() == "Propagating eigenvector...")
    with gzip.open(os.path.join(d, "expected.txt.gz"), "wt") as f:
        f.write("\n".join(lines[k - 1:]) + "\n")
    # MAKECST's lines, for the CPU test of the unit conversion
    with open(os.path.join(d, "constants.txt"), "w") as f:
        i = lines.index(" Initial potential:")
        j = lines.index(" Units converted.")
        f.write("\n".join(lines[i:j - 1]) + "\n")


def psod_cases():
    vmeta = dict(absorb="VOPTIC_POLIN", voi=[-0.02, 2.0], al=1.6, ar=2.2)
    smeta = dict(absorb="SMOOTHW", voi=[0.05, 1.0], al=1.55, ar=2.3)
    return {"morse1d_psod": case_morse1d("morse1d_psod", ".PSOD", "", {}),
            "morse1d_psod_voptic": case_morse1d("morse1d_psod_voptic", ".PSOD", VOPTIC, vmeta),
            "morse1d_psod_smooth": case_morse1d("morse1d_psod_smooth", ".PSOD", SMOOTH, smeta),
            "morse2d_psod": case_morse2d("morse2d_psod", ".PSOD")}


def save(cases, manifest):
    for name, (meta, arrays) in cases.items():
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
        manifest[name] = meta
        print(name, {k: getattr(a, "shape", None) for k, a in arrays.items()})
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


def main():
    if not os.path.exists(BIN):
        sys.exit("eSPec executable not found at " + BIN)
    if "--calc2d-only" in sys.argv:
        for name in CALC2D:
            case_calc2d(name)
        return
    if "--makecst-only" in sys.argv:
        case_makecst()
        return
    if "--collision-only" in sys.argv:
        for name in COLLISION_DECKS:
            case_collision(name)
        return
    if "--ti-only" in sys.argv:
        for name, deck in ti_decks().items():
            case_ti(name, deck)
        return
    if "--reftests-only" in sys.argv:
        picked = [a for a in sys.argv[1:] if a in map(str, REFTESTS)] or REFTESTS
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(4) as ex:
            list(ex.map(case_reftest, picked))
        return
    if "--decks-only" in sys.argv:
        names = [a for a in sys.argv[1:] if a in DECK_CASES] or list(DECK_CASES)
        for name in names:
            case_deck(name)
        return
    if "--psod-only" in sys.argv:
        with open(os.path.join(OUT, "manifest.json")) as f:
            manifest = json.load(f)
        save(psod_cases(), manifest)
        return
    if "--text-only" in sys.argv:  # only the *_partial.txt files
        vmeta = dict(absorb="VOPTIC_POLIN", voi=[-0.02, 2.0], al=1.6, ar=2.2)
        case_morse1d("morse1d_spo", ".PFSPO", "", {})
        case_morse1d("morse1d_sod", ".PFSOD", "", {})
        case_morse1d("morse1d_spo_voptic", ".PFSPO", VOPTIC, vmeta)
        case_sil_order_text(".YES")
        case_sil_order_text(".NO")
        case_test8_text()
        return
    case_sil_order_text(".YES")
    case_sil_order_text(".NO")
    case_test8_text()
    cases = {}
    cases["test8"] = case_test8()
    cases["test4"] = case_test4()
    for prop, tag in [(".PFSOD", "sod"), (".PFSPO", "spo"), (".PSIL", "sil")]:
        cases[f"morse1d_{tag}"] = case_morse1d(f"morse1d_{tag}", prop, "", {})
    vmeta = dict(absorb="VOPTIC_POLIN", voi=[-0.02, 2.0], al=1.6, ar=2.2)
    smeta = dict(absorb="SMOOTHW", voi=[0.05, 1.0], al=1.55, ar=2.3)
    for prop, tag in [(".PFSOD", "sod"), (".PFSPO", "spo")]:
        cases[f"morse1d_{tag}_voptic"] = case_morse1d(f"morse1d_{tag}_voptic", prop, VOPTIC, vmeta)
    for prop, tag in [(".PFSOD", "sod"), (".PFSPO", "spo"), (".PSIL", "sil")]:
        cases[f"morse1d_{tag}_smooth"] = case_morse1d(f"morse1d_{tag}_smooth", prop, SMOOTH, smeta)
    for prop, tag in [(".PSIL", "sil"), (".PFSPO", "spo"), (".PFSOD", "sod")]:
        cases[f"morse2d_{tag}"] = case_morse2d(f"morse2d_{tag}", prop)
    cases.update(psod_cases())
    save(cases, {})
    for name in DECK_CASES:
        case_deck(name)
    for i in REFTESTS:
        case_reftest(i)
    for name in CALC2D:
        case_calc2d(name)
    for name, deck in ti_decks().items():
        case_ti(name, deck)
    for name in COLLISION_DECKS:
        case_collision(name)
    case_makecst()


if __name__ == "__main__":
    main()
