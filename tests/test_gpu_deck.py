"""Whole eSPec input decks run by the deck driver (espec_run_deck) on the GPU
against the shipped executable's output for the same decks and files
(tests/golden/deck_*/expected.txt, from the propagation to the end): every
line of text identical; every printed number within one unit of its last
printed digit (both sides rounded FP64 values; E-format fields relative).
.PSIL and .PPSIL decks get 4e-7 more: the reference bisects the eigenvalues of its
Krylov matrices only to ABSTOL = 1e-6 (espec.f:157), which moves C(t) by a
few 1e-8 over these runs (the same allowance as the PLNZ drop-in's test).
For .PSIL the executable's total correlation is corrupted (it stores C(t)
in LNZVC columns MP+1, MP+2 past the LMTREORT columns of its array, where
scratch data overwrite samples); there the driver's table is checked against
the mirror assembly of the C samples in its own partial table instead."""
import gzip
import os
import re

import numpy as np
import pytest

from espec_b200 import deck as D

import golden_cases as G

pytestmark = pytest.mark.gpu

DECKS = ["deck_spo_hwhm", "deck_psod_voptic", "deck_sil_smooth", "deck_sil_2d", "deck_ppsod",
         "deck_ppsod_proj", "deck_ppsil", "deck_ppsil_proj", "deck_ppsod_2d", "deck_ppsil_2d",
         "deck_ppsod_ggaus", "deck_ppsod_sin2"]
NUM = re.compile(r"^-?(\d+\.?\d*|\.\d+)([EeDd][-+]?\d+)?$")


def unit_of(tok):
    """One unit of the last printed digit of a number field."""
    if "E" in tok.upper():
        mant, ex = re.split("[EeDd]", tok)
        dec = len(mant.split(".")[1]) if "." in mant else 0
        return 10.0 ** (int(ex) - dec)
    return 10.0 ** -(len(tok.split(".")[1]) if "." in tok else 0)


def is_row(line, ncol):
    t = line.split()
    return len(t) == ncol and all(NUM.match(x) for x in t)


def compare(have, want, slack=0.0):
    exact = 0
    assert len(have) == len(want), (len(have), len(want))
    for h, w in zip(have, want):
        if h == w:
            exact += 1
            continue
        ht, wt = h.split(), w.split()
        assert len(ht) == len(wt), (h, w)
        for a, b in zip(ht, wt):
            if a == b:
                continue
            assert NUM.match(a) and NUM.match(b), (h, w)
            da, db = float(a.replace("D", "E")), float(b.replace("D", "E"))
            assert abs(da - db) <= 1.01 * unit_of(b) + slack, (h, w)
    return exact


MARKS = ("Propagating eigenvector...", "Getting correlation function...",
         "Generating initial potential...")


def run_and_read(capfd, d, tmp=None):
    """The driver's output for the deck in directory d, from the line before
    the last 'Propagating eigenvector...' (for .ONLYSPEC 'Getting correlation
    function...', for .PES 'Generating initial potential...'), and the
    executable's.  Gzipped input files
    beside the deck are unpacked with it into tmp."""
    deck = os.path.join(d, "input.spc")
    packed = [f for f in os.listdir(d) if f.endswith(".gz") and f != "expected.txt.gz"]
    if packed:
        with open(deck) as f:
            (tmp / "input.spc").write_text(f.read())
        for name in packed:
            with gzip.open(os.path.join(d, name), "rt") as f:
                (tmp / name[:-3]).write_text(f.read())
        deck = str(tmp / "input.spc")
    capfd.readouterr()
    D.run(deck)
    out, err = capfd.readouterr()
    assert err == ""
    lines = out.split("\n")
    i = max(k for k, l in enumerate(lines) if l.strip() in MARKS)
    if os.path.exists(os.path.join(d, "expected.txt")):
        with open(os.path.join(d, "expected.txt")) as f:
            want = f.read().split("\n")
    else:
        with gzip.open(os.path.join(d, "expected.txt.gz"), "rt") as f:
            want = f.read().split("\n")
    return lines[i - 1:], want


@pytest.mark.parametrize("name", DECKS)
def test_deck_matches_executable(capfd, name):
    have, want = run_and_read(capfd, os.path.join(G.GOLDEN, name))
    if "_sil" not in name:
        exact = compare(have, want, slack=4e-7 if "ppsil" in name else 0.0)
        assert exact >= 0.9 * len(want), (exact, len(want))
        return
    check_sil(have, want, 4e-7)


# The reference's own test decks (ttests/input.test<i>): an analytic .1D
# potential, the initial state computed (.CALC) and propagated on the final
# potential for 125 thousand to 3 million steps.  Allowances beyond one unit
# of the last printed digit, measured:
#   .PFSPO, .PFSOD (tests 6, 12, 10): the executable's C(t) drifts from the
#     oracle's restatements of spofft.f / sodfft.f (which the GPU matches to
#     print precision) by a phase growing linearly with t: 3e-7 (.PFSPO) and
#     6.3e-6 (.PFSOD, N = 250) after 2.5 million steps; the cause is not
#     pinned (fft3d.f's single-precision constants are a candidate);
#   .PSIL, .PPSIL (tests 13, 14): the executable bisects the eigenvalues of
#     its Krylov matrices to ABSTOL = 1e-6 only, so its norm falls by 3e-6
#     over the 125 thousand steps and C(t) moves by up to 4.5e-6; its total
#     correlation is corrupted (samples overwritten, see check_sil).
# .PSOD and .PPSOD (tests 9, 11) need none, nor test 2 (.PPSOD, six
# populations on computed states, HWHM shifted by the computed E1I) and test
# 3 (.PPSOD, a .GGAUS pulse on the dipole file dipol2.inp, six populations;
# 40 fs of its 2000), both run with .MTRXDIAG: their own .LANCZS gives the
# executable ghost eigenvalues.
REFTESTS = {"reftest9": 0.0, "reftest10": 8e-6, "reftest11": 0.0, "reftest12": 4e-7,
            "reftest6": 4e-7, "reftest13": 5e-6, "reftest14": 5e-6, "reftest2_mtrxdiag": 0.0,
            "reftest3_short": 0.0,
            # 2D .CALC decks (tests/golden/make_golden.py CALC2D): .MTRXDIAG states
            # of a 32 x 32 grid, 1920 .PSIL steps (the ABSTOL bisection again, on
            # Krylov spectra ten times wider: 7e-7 in C(t), 1e-6 in the norm) and
            # 1920 .PSOD steps
            "calc2d_ohs_psil": 1.5e-6, "calc2d_morse_psod": 0.0,
            # test 8: .ONLYSPEC on the correlation function of an old output
            # (ttests/correl8.inp), HWHM and the spectrum; test 4: .PSIL from a
            # .FILE (the allowance of test 13); test 15: .PES, the 2D .LEPS_CC
            # potential printed on 200 x 180 points
            "reftest8": 0.0, "reftest4": 5e-6, "reftest15": 0.0,
            # .COLLISION (make_golden.py COLLISION): a complex Gaussian wave
            # packet, 100 thousand steps; .PSOD with the reference's restart
            # copy (its norm drifts to INFO = 1), every line identical; .PFSPO:
            # the packet's momentum puts weight on high k, where the in-place
            # kinetic multiply (spofft.f:150-153) is far from unitary, and the
            # executable drifts from the oracle's restatement (which the GPU
            # matches to print precision) by up to 1.7e-4 in C(t) over the 20 fs
            "collision_psod": 0.0, "collision_pfspo": 3e-4}
SIL_DECKS = ("reftest13", "reftest14", "calc2d_ohs_psil", "reftest4")


@pytest.mark.parametrize("name", sorted(REFTESTS))
def test_reference_test_deck(capfd, tmp_path, name):
    have, want = run_and_read(capfd, os.path.join(G.GOLDEN, name), tmp_path)
    if name in SIL_DECKS:
        check_sil(have, want, REFTESTS[name])
    else:
        compare(have, want, slack=REFTESTS[name])


def check_sil(have, want, slack):
    """Partial table within slack; the executable's total correlation and
    spectrum are not comparable (LNZVC columns overwritten), so the driver's
    total correlation is checked against the mirror assembly of its own
    partial table, and the text lines of the rest against the executable's."""
    k = have.index(" Correlation Function:")
    assert want.index(" Correlation Function:") == k and len(have) == len(want)
    compare(have[:k], want[:k], slack=slack)
    for h, w in zip(have[k:], want[k:]):  # the text lines of the rest
        if not (w.split() and all(NUM.match(t) or set(t) == {"*"} for t in w.split())):
            assert h == w, (h, w)
    # total correlation: C(-t) = C(t)*, 2^MF samples from the partial table
    # (PPLNZ's 1D table, "Auto-correlation function:", prints Cr, Ci in
    # columns 4, 5 with five decimals; PLNZ's in columns 3, 4 with seven)
    j = [i for i, l in enumerate(have) if l.strip() in ("Partial auto-correlation function:",
                                                        "Auto-correlation function:")][0]
    pulse = have[j].strip() == "Auto-correlation function:"
    ncol = max(len(l.split()) for l in have[j + 3:k])
    part = np.array([[float(x) for x in l.split()] for l in have[j + 3:k] if is_row(l, ncol)])
    corr = np.array([[float(x) for x in l.split()] for l in have[k + 3:] if is_row(l, 3)])
    mc = len(corr) // 2
    c = part[:mc, 3] + 1j * part[:mc, 4] if pulse else part[:mc, 2] + 1j * part[:mc, 3]
    tol = 0.51e-5 + 0.51e-7 if pulse else 1.01e-7
    full = np.concatenate([[np.conj(c[mc - 1])], np.conj(c[1:mc][::-1]), c])
    assert np.max(np.abs(corr[:, 1] - full.real)) <= tol
    assert np.max(np.abs(corr[:, 2] - full.imag)) <= tol


def test_scan_equals_one_run_per_file(tmp_path, capfd):
    """Three .FILE inputs (the fixture's and two displaced Gaussians) through
    espec_run_scan: each job's correlation and spectrum blocks are the text the
    single-deck driver prints for that file."""
    src = os.path.join(G.GOLDEN, "deck_spo_hwhm")
    deck = open(os.path.join(src, "input.spc")).read()
    lines = open(os.path.join(src, "wf_pot.inp")).read().split("\n")
    n = 256
    x = np.array([float(l.split()[0]) for l in lines[1:1 + n]])
    files = ["wf_pot.inp"]
    (tmp_path / "wf_pot.inp").write_text("\n".join(lines))
    for k, x0 in enumerate((1.7, 1.95)):
        psi = np.exp(-((x - x0) ** 2) / (2 * 0.18 ** 2))
        psi /= np.sqrt(np.sum(psi ** 2))
        body = [lines[0]] + [f" {repr(float(a))}   {repr(float(b))}" for a, b in zip(x, psi)]
        body += lines[1 + n:]
        name = f"wf_{k}.inp"
        (tmp_path / name).write_text("\n".join(body))
        files.append(name)
    (tmp_path / "input.spc").write_text(deck)
    capfd.readouterr()
    D.run_scan(tmp_path / "input.spc", files, tmp_path / "job")
    capfd.readouterr()
    for k, f in enumerate(files, 1):
        (tmp_path / f"single_{k}.spc").write_text(deck.replace("wf_pot.inp", f))
        D.run(tmp_path / f"single_{k}.spc")
        out = capfd.readouterr().out
        i = out.index(" \n Correlation Function:")
        j = out.index(" \n Spectrum:")
        crl = (tmp_path / f"job{k}.crl").read_text()
        spc = (tmp_path / f"job{k}.spc").read_text()
        assert out[i:].startswith(crl)
        assert spc == out[j:j + len(spc)]
        assert out[j + len(spc):].startswith(" Spectrum done.")


# The time-independent formalism (tests/golden/ti_*): .ENERGY and .SPECTRUM
# .TI (SPECTRUMTI's Franck-Condon table) on the surfaces of reference test 12
# and on a 2D pair.  The executable's eigenvalues are DSPEVX bisections to
# ABSTOL = 1e-6 (the same state prints 0.440579E-02 or 0.440584E-02 with
# different *NIST ranges; the converged value is 0.440574E-02), so eigenvalues
# and the transition energies E get 1.1e-6; the amplitudes are compared in
# magnitude (an eigenvector's sign is arbitrary) and, with the Franck-Condon
# factors, to one unit of the last printed digit.
TI_DECKS = ["ti_energy_ohs", "ti_spectrum_ohs", "ti_spectrum_2d_ohs"]


@pytest.mark.parametrize("name", TI_DECKS)
def test_time_independent_deck(capfd, name):
    d = os.path.join(G.GOLDEN, name)
    capfd.readouterr()
    D.run(os.path.join(d, "input.spc"))
    out, err = capfd.readouterr()
    assert err == ""
    lines = out.split("\n")
    i = min(k for k, l in enumerate(lines)
            if l.strip() == "Calculating eigenvalue(s) and eigenvector(s)")
    have = lines[i - 1:]
    with open(os.path.join(d, "expected.txt")) as f:
        want = f.read().split("\n")

    def unsign_amplitudes(rows):
        out, spec = [], False
        for l in rows:
            t = l.split()
            if l.strip() == "Spectrum:":
                spec = True
            if spec and len(t) == 6 and t[4] == "->":
                l = l.replace(t[1], t[1].lstrip("-"), 1)
            out.append(l)
        return out

    compare(unsign_amplitudes(have), unsign_amplitudes(want), slack=1.1e-6)
