"""Run an eSPec input deck through the GPU propagators (espec_run_deck).

    python -m espec_b200.deck path/to/input.spc
    python -m espec_b200.deck path/to/input.spc data1.inp data2.inp ... out_prefix

runs espec.f's driver for one packet: a .FILE potential with its .GETR
eigenvector, or analytic 1D/2D potentials with the initial states computed
(.CALC) on the GPU; the time-dependent propagators (.PFSPO, .PFSOD, .PSIL,
.PSOD, and .PPSOD / .PPSIL with a laser pulse; absorbers, total correlation,
HWHM, spectrum), the time-independent formalism (.ENERGY, .SPECTRUM .TI),
.PES and .ONLYSPEC, printing what espec.x prints; other decks are refused with
the reason.
"""
import sys

from . import _native as N


def run(path):
    """Runs the deck; raises EspecError with the reason when it is refused or
    a device call fails."""
    N.check(N.load().espec_run_deck(str(path).encode()), "espec_run_deck")


def run_scan(path, files, out_prefix):
    """The deck over several .FILE inputs as one batched GPU run (1D .PFSPO or
    .PFSOD): writes <out_prefix><k>.crl and <out_prefix><k>.spc, k = 1.."""
    import ctypes as C

    arr = (C.c_char_p * len(files))(*[str(f).encode() for f in files])
    N.check(N.load().espec_run_scan(str(path).encode(), len(files), arr, str(out_prefix).encode()),
            "espec_run_scan")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) == 0 or len(argv) == 2:
        sys.stderr.write("usage: python -m espec_b200.deck input.spc [data.inp ... out_prefix]\n")
        return 2
    try:
        if len(argv) == 1:
            run(argv[0])
        else:
            run_scan(argv[0], argv[1:-1], argv[-1])
    except N.EspecError as e:
        sys.stderr.write(str(e) + "\n")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
