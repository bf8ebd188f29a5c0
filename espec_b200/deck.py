"""Run an eSPec input deck through the GPU propagators (espec_run_deck).

    python -m espec_b200.deck path/to/input.spc

covers the time-dependent part of espec.f for one packet with a .FILE
potential and its .GETR eigenvector (.PFSPO, .PFSOD, .PSIL, .PSOD, absorbers,
total correlation, HWHM, spectrum) and prints what espec.x prints from
"Propagating eigenvector..." on; other decks are refused with the reason.
"""
import sys

from . import _native as N


def run(path):
    """Runs the deck; raises EspecError with the reason when it is refused or
    a device call fails."""
    N.check(N.load().espec_run_deck(str(path).encode()), "espec_run_deck")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        sys.stderr.write("usage: python -m espec_b200.deck input.spc\n")
        return 2
    try:
        run(argv[0])
    except N.EspecError as e:
        sys.stderr.write(str(e) + "\n")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
