"""The deck driver's reading of eSPec input decks (espec_b200/csrc/deck.cpp),
on the CPU: what it does not cover is refused with the reason before any
device work, a .FILE that is missing or short is reported, and the unit
conversion of analytic potentials (MAKECST) prints the executable's
constants."""
import os

import pytest

from espec_b200 import _native as N
from espec_b200 import deck as D

HERE = os.path.dirname(os.path.abspath(__file__))
BASE = open(os.path.join(HERE, "golden", "deck_spo_hwhm", "input.spc")).read()


def refused(tmp_path, text, files=None):
    p = tmp_path / "input.spc"
    p.write_text(text)
    for name, body in (files or {}).items():
        (tmp_path / name).write_text(body)
    with pytest.raises(N.EspecError) as e:
        D.run(p)
    return str(e.value)


@pytest.mark.parametrize("old,new,why", [
    # an analytic potential turns *INIEIGVC into .CALC; the deck has no grid
    (".FILE\nwf_pot.inp", ".MORSE\n1.1 1943.8 13.7 1.0/\n1.2 1629.2 17.7 1.0/", "*GRID_RANGES"),
    (".GETR", ".CALC", ".GETR"),
    (".PFSPO", ".P2PABM", "propagator"),
    (" 0.0  0.3096171935104  0.00120944216215/", " 0.0  0.3096171935104  0.0/", "DT must be"),
    (".1D\n 256/", ".2DC\n 16 16/", "*DIMENSION"),
    ("*TPTRANS\n.ONE", "*TPTRANS\n.ALL", "one propagated state"),
    ("*PRPGSTATE\n 0/", "*PRPGSTATE\n 1/", "*PRPGSTATE 0"),
    ("**TD", "**COLLISION\n**TD", "section **COLLISION"),
    ("**TD", "**TI\n*QUANTUM_FOO\n 1.0/\n**TD", "keyword *QUANTUM_FOO"),
    ("*PRPTOL", "*PULSE_AND_DIPOLE\n.GAUS\n*PRPTOL", "*PULSE_AND_DIPOLE"),
    ("*PRPTOL", "*PULSE_AND_DIPOLE\n.LASER\n 1 2 3 4 5/\n.NULL\n*PRPTOL", "pulse is not known"),
    ("*PRPTOL", "*PULSE_AND_DIPOLE\n.GAUS\n 1 2 3 4 5/\n.GET\ndm.inp\n*PRPTOL", "dipole moment .GET"),
    ("*PRPTOL", "*PULSE_AND_DIPOLE\n.GAUS\n 1 2 3 4 5/\n.EXP\n 0.5/\n*PRPTOL", "constants"),
])
def test_uncovered_decks_are_refused(tmp_path, old, new, why):
    assert old in BASE
    msg = refused(tmp_path, BASE.replace(old, new))
    assert why in msg, msg


def test_ppsod_projections(tmp_path):
    """rdinput.f:659-660 with one state from .GETR: NPR + KP > 1 lowers NPR
    by one; what is left of NPR would project on states the deck does not
    have."""
    text = BASE.replace(".PFSPO", ".PPSOD")
    for npr_kp in ("3 1", "2 1", "3 0"):
        msg = refused(tmp_path, text.replace("*PRPTOL", f"*NPROJECTIONS\n {npr_kp}/\n*PRPTOL"))
        assert "*NPROJECTIONS" in msg, (npr_kp, msg)
    # NPR = 1, KP = 1 leaves none; NPR = 2, KP = 0 leaves one on LNZVC(., 1):
    # the deck passes the reading and stops at its (absent) .FILE
    for npr_kp in ("1 1", "2 0"):
        msg = refused(tmp_path, text.replace("*PRPTOL", f"*NPROJECTIONS\n {npr_kp}/\n*PRPTOL"))
        assert "cannot be opened" in msg, (npr_kp, msg)
    # PPLNZ prints NPR - 1 projections after |C|^2
    text = BASE.replace(".PFSPO\n 0.0  0.3096171935104  0.00120944216215/",
                        ".PPSIL\n 0.0  0.3096171935104  0.00120944216215 10/")
    assert text != BASE
    for npr_kp, why in (("3 0", "cannot be opened"), ("4 0", "*NPROJECTIONS"),
                        ("3 1", "*NPROJECTIONS"), ("2 1", "cannot be opened")):
        msg = refused(tmp_path, text.replace("*PRPTOL", f"*NPROJECTIONS\n {npr_kp}/\n*PRPTOL"))
        assert why in msg, (npr_kp, msg)


PULSE_BLOCKS = ["*PULSE_AND_DIPOLE\n.GAUS\n 5.0D7  0.1  2.5  0.15  0.0/\n.EXP\n 0.5 0.3 0.0/",
                "*PULSE_AND_DIPOLE\n.GGAUS\n 3D11 0.08 2.5 0.12 0.3 2/\n.CONST\n 1.0/",
                "*PULSE_AND_DIPOLE\n.SIN2\n 6D7 0.2 3.0 0.05 0.0/\n.NULL",
                "*PULSE_AND_DIPOLE\n.NONE\n 0 0 0/\n.NONE\n 0.0/"]


@pytest.mark.parametrize("prop", [".PPSOD\n 0.0  0.3096171935104  0.00120944216215/",
                                  ".PPSIL\n 0.0  0.3096171935104  0.00120944216215 10/"])
@pytest.mark.parametrize("block", PULSE_BLOCKS)
def test_pulse_blocks_are_read(tmp_path, prop, block):
    """rdinput.f:549-578: each pulse shape's parameter record and each
    dipole form's record; a deck that reads through stops at its (absent)
    .FILE, before any device work."""
    text = BASE.replace(".PFSPO\n 0.0  0.3096171935104  0.00120944216215/", prop)
    text = text.replace("*PRPTOL", block + "\n*PRPTOL")
    assert text != BASE
    msg = refused(tmp_path, text)
    assert "cannot be opened" in msg, msg


@pytest.mark.parametrize("block,why", [
    ("*PULSE_AND_DIPOLE\n.GGAUS\n 3D11 0.08 2.5 0.12 0.3/\n.NULL", "KL"),
    ("*PULSE_AND_DIPOLE\n.SIN2\n 6D7 0.2 3.0/\n.NULL", "TD"),
    ("*PULSE_AND_DIPOLE\n.GAUS\n 1 2 3 4 5/\n.EXP+\n 0.5 0.3/", "dipole .EXP+"),
    ("*PULSE_AND_DIPOLE\n.GAUS\n 1 2 3 4 5/\n.LINEAR\n 0.5/", "wasn't found"),
])
def test_pulse_blocks_refused(tmp_path, block, why):
    msg = refused(tmp_path, BASE.replace("*PRPTOL", block + "\n*PRPTOL"))
    assert why in msg, msg


def test_missing_and_short_files(tmp_path):
    assert "cannot be opened" in refused(tmp_path, BASE)
    short = "# Eigenvector:\n 0.5 0.1\n 0.6 0.2\n"
    assert "reading file error" in refused(tmp_path, BASE, {"wf_pot.inp": short})


def test_final_time_not_adequate_for_fft(tmp_path, capfd):
    text = BASE.replace("*CHANGE\n.YES", "*CHANGE\n.NO").replace("0.3096171935104", "0.31")
    src = open(os.path.join(HERE, "golden", "deck_spo_hwhm", "wf_pot.inp")).read()
    msg = refused(tmp_path, text, {"wf_pot.inp": src})
    assert "not adequate for FFT" in msg
    assert "<<<>>> Final time is not adequate for FFT <<<>>>" in capfd.readouterr().out


def test_final_time_warning_text(tmp_path, capfd):
    """*CHANGE .YES with a TF that does not fit 2^MF samples: the warning
    line as the executable prints it (its list-directed REAL*8 is 1PG23.15E3;
    text taken from espec_v07.x on this deck with TF = 0.3101).  Printed
    before any device work, so the check runs with or without a GPU."""
    src = os.path.join(HERE, "golden", "deck_spo_hwhm")
    (tmp_path / "wf_pot.inp").write_text(open(os.path.join(src, "wf_pot.inp")).read())
    (tmp_path / "input.spc").write_text(BASE.replace("0.3096171935104", "0.3101"))
    try:
        D.run(tmp_path / "input.spc")
    except N.EspecError:
        pass  # no device here: the propagation itself fails after the warning
    out = capfd.readouterr().out.split("\n")
    assert " -> Warning! Final time changed to  0.309617193510400     " in out


# the reference's test deck 6 (ttests/input.test6) with MF lowered, and the
# constants its executable prints for it (espec_v07.x, "Initial potential:" /
# "Final potential:" lines)
CALC = """*** eSPec input file ***
**MAIN
*DIMENSION
.1D
 256/
*POTENTIAL
.MORSE
 1.14600  1943.79  13.71  1.0/
 1.21100  1629.23  17.74  1.0/
*GRID_RANGES
 0.5  2.8/
*MASS
 7.49D0/
*TPCALC
.SPECTRUM
.TD
*INIEIGVC
.CALC
*CHANGE
.YES
**TI
*TPDIAG
.LANCZS
*NIST
 1  0/
*ABSTOL
 1D-6/
**TD
*PROPAG
.PFSPO
 0.0  0.0512  2D-4/
*PRPGSTATE
 0/
*TPTRANS
.ONE
**SPECTRUM
*FOURIER
 8/
*WINDOWING
.SG
 1D-5/
**END
"""
CALC_CONSTANTS = [
    " Re_1/a.u. = 0.216563E+01; alpha_1/a.u. = 0.131080E+01; D_1/a.u. = 0.313919E+00",
    " Re_1/a.u. = 0.228846E+01; alpha_1/a.u. = 0.149106E+01; D_1/a.u. = 0.170438E+00"]


def run_calc(tmp_path, text):
    """Runs a .CALC deck; without a GPU it stops at the first device buffer,
    after the unit conversion.  Returns the error message or None."""
    p = tmp_path / "input.spc"
    p.write_text(text)
    try:
        D.run(p)
    except N.EspecError as e:
        return str(e)
    return None


def test_calc_morse_constants(tmp_path, capfd):
    """MAKECST of .MORSE (makecst.f:134-157): Re / A0A, alpha and D from the
    frequency and the anharmonic constant; the two lines the executable
    prints for the reference's test deck 6."""
    msg = run_calc(tmp_path, CALC)
    assert msg is None or "device memory" in msg, msg
    out = capfd.readouterr().out.split("\n")
    i = out.index(" Initial potential:")
    assert out[i + 1] == CALC_CONSTANTS[0]
    assert out[i + 2] == " Final potential:"
    assert out[i + 3] == CALC_CONSTANTS[1]
    assert " -> Warning step bigger than  1.000000000000000E-002  a.u. !" in out


def test_calc_ohs_constants(tmp_path, capfd):
    """.OHS (makecst.f:83-88): the constants the executable prints for the
    reference's test decks 9-14."""
    text = CALC.replace(".MORSE\n 1.14600  1943.79  13.71  1.0/\n 1.21100  1629.23  17.74  1.0/",
                        ".OHS\n 1.14600  1943.79/\n 1.21100  1629.23/")
    msg = run_calc(tmp_path, text)
    assert msg is None or "device memory" in msg, msg
    out = capfd.readouterr().out.split("\n")
    assert " Re_1/a.u. = 0.216563E+01; K_1/a.u. = 0.107875E+01;" in out
    assert " Re_1/a.u. = 0.228846E+01; K_1/a.u. = 0.757856E+00;" in out


@pytest.mark.parametrize("old,new,why", [
    (".1D\n 256/", ".3D\n 16 16 16/", ".2D grids"),
    (".1D\n 256/", ".2D\n 64 64/", "XI < XF"),
    ("*NIST\n 1  0/", "*NIST\n 3  1/", "*PRPGSTATE must be one of"),
    ("*NIST\n 1  0/", "*NIST\n 17  0/", "16 lowest states"),
    (".LANCZS\n", ".JACOBI\n", "eigenvalue(s) and eigenvector(s)"),
    (".MORSE\n", ".DMORSE\n", "no unit conversion"),
    (".MORSE\n", ".WELL\n", "not a form of .1D grids"),
    (" 0.5  2.8/", " 2.8  0.5/", "XI < XF"),
    (" 1.21100  1629.23  17.74  1.0/\n", "", "missing record of *POTENTIAL"),
    (" 256/", " 20/", "grid step is above 4e-2"),
])
def test_calc_refusals(tmp_path, old, new, why):
    """What the .CALC path does not cover, or where the executable stops, is
    refused before any device work."""
    assert old in CALC
    msg = run_calc(tmp_path, CALC.replace(old, new))
    assert msg is not None and why in msg, msg


def test_calc_projections_on_computed_states(tmp_path):
    """rdinput.f:659-660 with NIS computed states: the populations PPSOD
    prints are on states KP+1..KP+NPR, which *NIST must provide."""
    text = CALC.replace(".PFSPO\n 0.0  0.0512  2D-4/", ".PPSOD\n 0.0  0.0512  2D-4/")
    text = text.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.PROPAGATION")
    # NPR + KP > NIS lowers NPR by NIS: 3 1 with NIS = 3 leaves none; 6 1
    # leaves 3 on states 2..4, one past the computed ones
    for nist, proj, ok in (("7  0", "6 1", True), ("3  0", "3 1", True), ("3  0", "2 1", True),
                           ("3  0", "6 1", False)):
        t = text.replace("*NIST\n 1  0/", f"*NIST\n {nist}/")
        t = t.replace("*TPTRANS", f"*NPROJECTIONS\n {proj}/\n*TPTRANS")
        msg = run_calc(tmp_path, t)
        if ok:
            assert msg is None or "device memory" in msg, (nist, proj, msg)
        else:
            assert msg is not None and "*NPROJECTIONS" in msg, (nist, proj, msg)


def test_dipole_file_is_read(tmp_path):
    """*PULSE_AND_DIPOLE .READ (rdinput.f:571-572, dipl.f:81-82): the dipole
    file's name is the record after .READ, relative to the deck; a missing
    file is reported after the deck's own .FILE is read, before any device
    work."""
    src = os.path.join(HERE, "golden", "deck_ppsod")
    text = open(os.path.join(src, "input.spc")).read()
    i = text.index("*PULSE_AND_DIPOLE")
    j = text.index("*", i + 1)
    pulse = "*PULSE_AND_DIPOLE\n.GAUS\n 5.0D7  0.1  2.5  0.15  0.0/\n.READ\nmu.inp\n"
    files = {"wf_pot.inp": open(os.path.join(src, "wf_pot.inp")).read()}
    msg = refused(tmp_path, text[:i] + pulse + text[j:], files)
    assert "dipole file" in msg and "mu.inp" in msg, msg


@pytest.mark.parametrize("name", ["calc2d_ohs_psil", "calc2d_morse_psod"])
def test_calc_2d_constants(tmp_path, capfd, name):
    """MAKECST's 2D branch (makecst.f:176-340): the lines the executable
    prints for the two 2D .CALC decks -- .OHS in cm^-1 with two masses, and a
    .MORSE pair, for which MAKECST has no 2D branch (the message; the
    constants stay in atomic units)."""
    d = os.path.join(HERE, "golden", name)
    msg = run_calc(tmp_path, open(os.path.join(d, "input.spc")).read())
    assert msg is None or "device memory" in msg, msg
    out = capfd.readouterr().out.split("\n")
    want = open(os.path.join(d, "constants.txt")).read().rstrip("\n").split("\n")
    i = out.index(" Initial potential:")
    assert out[i:i + len(want)] == want


def test_onlyspec_reads_and_prints_the_correlation(tmp_path, capfd):
    """.ONLYSPEC (espec.f:1596-1626, getcorr.f): the reference's test deck 8
    reads the 2^MF rows after " Correlation Function:" of an old output and
    prints them again as the executable does (DTF from the first two times,
    TF = last time + DTF); the HWHM and spectrum that follow run on the GPU
    (tests/test_gpu_deck.py)."""
    import gzip
    d = os.path.join(HERE, "golden", "reftest8")
    (tmp_path / "input.spc").write_text(open(os.path.join(d, "input.spc")).read())
    with gzip.open(os.path.join(d, "correl8.inp.gz"), "rt") as f:
        (tmp_path / "correl8.inp").write_text(f.read())
    try:
        D.run(tmp_path / "input.spc")
    except N.EspecError:
        pass
    out = capfd.readouterr().out.split("\n")
    with gzip.open(os.path.join(d, "expected.txt.gz"), "rt") as f:
        want = f.read().split("\n")
    i, j = out.index(" Correlation function got."), want.index(" Correlation function got.")
    k = want.index(" Half-width at half-maximum applied.") - 2  # the HWHM message
    assert out[i:i + (k - j)] == want[j:k]


def test_time_independent_decks_are_read(tmp_path):
    """.ENERGY and .SPECTRUM .TI (rdinput.f:139-149, *NFST of rdinput.f:375-377):
    no propagator is needed; the .TI spectrum needs final states and computed
    ones; a deck that reads through stops at the first device buffer."""
    energy = CALC.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.ENERGY")
    msg = run_calc(tmp_path, energy.replace(".PFSPO\n", ".NULL\n"))
    assert msg is None or "device memory" in msg, msg
    ti = CALC.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.SPECTRUM\n.TI")
    msg = run_calc(tmp_path, ti)
    assert msg is not None and "*NFST" in msg, msg
    msg = run_calc(tmp_path, ti.replace("*NIST\n 1  0/", "*NIST\n 1  0/\n*NFST\n 4  0/"))
    assert msg is None or "device memory" in msg, msg
    msg = run_calc(tmp_path, CALC.replace("*TPCALC\n.SPECTRUM\n.TD", "*TPCALC\n.SPECTRUM\n.XX"))
    assert msg is not None and ".TD and .TI" in msg, msg


def test_keywords_match_by_prefix(tmp_path, capfd):
    """rdinput.f tests keyword lines by prefix: the reference's test deck 15
    writes *MASSES, *MASS_FACTORS and *GRID_RANGES_au (ranges in bohr).  It
    reads through (.PES, the 2D .LEPS_CC_Dalpha_au potential) to the first
    device buffer, printing MAKECST's lines as the executable does."""
    d = os.path.join(HERE, "golden", "reftest15")
    msg = run_calc(tmp_path, open(os.path.join(d, "input.spc")).read())
    assert msg is None or "device memory" in msg, msg
    out = capfd.readouterr().out.split("\n")
    i = out.index(" Initial potential:")
    assert out[i + 1:i + 7] == [
        " These parameters were already inputed in a.u.",
        " Re_1/a.u. = 0.140200E+01; alpha_1/a.u. = 0.102700E+01; D_1/a.u. = 0.174430E+00",
        " Re_2/a.u. = 0.140200E+01; alpha_2/a.u. = 0.102700E+01; D_2/a.u. = 0.174430E+00",
        " Re_3/a.u. = 0.140200E+01; alpha_3/a.u. = 0.102700E+01; D_3/a.u. = 0.174430E+00",
        " a = 0.3000E+00; b = 0.5000E-01; c = 0.5000E-01",
        " Angle (rad) =   3.14159265358979     "]


def test_collision_decks_are_read(tmp_path):
    """.COLLISION (rdinput.f:141-143, 384-419; espec.f:849-864): a 1D wave
    packet on an analytic potential reads through to the first device buffer;
    other forms are refused."""
    d = os.path.join(HERE, "golden", "collision_psod")
    text = open(os.path.join(d, "input.spc")).read()
    msg = run_calc(tmp_path, text)
    assert msg is None or "device memory" in msg, msg
    msg = run_calc(tmp_path, text.replace(" 0.1/\n", " 0.0/\n"))
    assert msg is not None and "*SIZE_OF_GAUSSIAN" in msg, msg
    msg = run_calc(tmp_path, text.replace(".1D\n 512/", ".2D\n 64 64/"))
    assert msg is not None and ".COLLISION" in msg, msg


def test_makecst_every_form(tmp_path, capfd):
    """MAKECST (makecst.f:82-340) for every named 1D and 2D form: the lines
    the executable prints for a .PES deck per form (tests/golden/
    makecst_lines.json), compared with the driver's, printed before any
    device work."""
    import json
    with open(os.path.join(HERE, "golden", "makecst_lines.json")) as f:
        cases = json.load(f)
    assert len(cases) >= 20
    for name, case in cases.items():
        capfd.readouterr()
        msg = run_calc(tmp_path, case["deck"])
        out = capfd.readouterr().out.split("\n")
        i = out.index(" Initial potential:")
        assert out[i:i + len(case["lines"])] == case["lines"], (name, msg)
