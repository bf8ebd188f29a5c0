"""CPU-side checks of the C-ABI library: it loads and exports every symbol
declared in include/espec_gpu.h.  No compute call is made."""
import ctypes as C
import os
import re

from espec_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "espec_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", src)
    keep = [n for n in names if n.startswith("espec_") or n.endswith("_")]
    return sorted(set(keep))


def test_library_loads_and_exports_declared_symbols():
    lib = N.load()
    declared = declared_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(N.EXPORTS) <= set(declared)
    assert lib.espec_version().startswith(b"espec_b200")


def test_errors_are_reported_without_a_device_call():
    lib = N.load()
    h = C.c_void_p()
    # invalid arguments are rejected on the host before any CUDA call
    rc = lib.espec_spo_create(C.byref(h), 0, None, None, None, 0.0, 0, 0, 0)
    assert rc == N.EINVAL
    assert b"null" in lib.espec_last_error()


def test_packet_sizes_refused_without_a_device_call():
    """Sizes outside the register FFT plans run FP64 only, even and up to the
    shared memory of one CTA (7252 points; 3626 for SOD); what is refused is
    refused before any CUDA call."""
    lib = N.load()
    cases = [(250, N.MIXED, N.SPO, b"mixed form"), (251, N.FP64, N.SPO, b"even sizes"),
             (8000, N.FP64, N.SPO, b"even sizes"), (4096, N.FP64, N.SOD, b"even sizes")]
    for n, prec, method, why in cases:
        h = C.c_void_p()
        npts = (C.c_int * 1)(n)
        sh, sm = (C.c_double * 1)(0.01), (C.c_double * 1)(1000.0)
        rc = lib.espec_prop_create(C.byref(h), 1, npts, sh, sm, C.c_double(0.1), method, prec,
                                   0, 0)
        assert rc == N.EINVAL, (n, prec, method)
        assert why in lib.espec_last_error(), (n, lib.espec_last_error())


def test_fortran_shim_binds_exported_drop_ins():
    """include/espec_gpu.f90 binds (bind(C)) only symbols the library exports,
    one per reference routine it replaces, with three hidden lengths each."""
    src = open(os.path.join(ROOT, "include", "espec_gpu.f90")).read()
    names = re.findall(r'bind\(C,\s*name="([a-z_]+)"\)', src)
    assert sorted(names) == ["plnz_", "psod_", "psodfft_", "pspofft_"]
    lib = N.load()
    for name in names:
        assert hasattr(lib, name), name
    assert src.count("integer(c_size_t), value :: dim_len, prtcrl_len, tpabsor_len") == 4
    for routine in ("espec_pspofft", "espec_psodfft", "espec_plnz", "espec_psod"):
        assert f"subroutine {routine}(" in src and f"end subroutine {routine}" in src
