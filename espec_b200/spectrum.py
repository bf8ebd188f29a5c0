"""Spectrum stage of eSPec on the GPU (FP64): total correlation assembly
(espec.f:1545-1576), HWHM (hwhm.f:59-77), the window, half swap and backward
FFTNT of SPECTRUMTD (spectrumtd.f:58-81, cfft.f:6-106), batched over packets.

`spectra()` works on device tensors (torch, complex128 or float64 pairs) --
typically the C(t) buffer a plan left on the device -- and returns the
2^mf-point results in FFTNT's natural order.  `hwhm()` and `spectrumtd()`
call the Fortran drop-ins hwhm_/spectrumtd_ on host arrays (the latter prints
the spectrum table as the reference does).
"""
import ctypes as C

import numpy as np

from . import _native as N


def spectra(c_dev, mf, dtf, tf, *, assemble=True, tal=None, de=0.0, window="SG", wp=1e-3,
            fftnt_sp=False, stream=None):
    """c_dev: torch complex128 device tensor [npk, ld] (C(t) samples when
    assemble, else 2^mf-point signals).  Returns torch complex128 [npk, 2^mf]."""
    import torch

    if c_dev.dtype != torch.complex128 or not c_dev.is_cuda or c_dev.dim() != 2:
        raise TypeError("c_dev must be a 2-D complex128 CUDA tensor")
    c_dev = c_dev.contiguous()
    npk, ld = c_dev.shape
    n = 1 << mf
    if assemble and ld < n // 2:
        raise ValueError("assembly needs 2^(mf-1) C(t) samples per packet")
    if not assemble and ld < n:
        raise ValueError("signals need 2^mf points per packet")
    lib = N.load()
    out = torch.empty((npk, n), dtype=torch.complex128, device=c_dev.device)
    wbytes = lib.espec_spectrum_work_bytes(npk, mf)
    work = torch.empty(max(1, (wbytes + 15) // 16), dtype=torch.complex128, device=c_dev.device)
    win = {"SG": 1, None: 0, "NONE": 0}[window]
    rc = lib.espec_spectrum_dev(npk, mf, c_dev.data_ptr(), ld, 1 if assemble else 0, float(dtf),
                                float(tf), -1.0 if tal is None else float(tal), float(de), win,
                                float(wp), N.Q_FFTNT_SP if fftnt_sp else 0, out.data_ptr(),
                                work.data_ptr(),
                                stream if stream is not None else
                                torch.cuda.current_stream(c_dev.device).cuda_stream)
    N.check(rc, "espec_spectrum_dev")
    return out


def hwhm(m, dt, tf, tal, de, u, v):
    """HWHM in place on float64 arrays u, v; returns TAL as the reference
    leaves it (scaled by 1.5192676, hwhm.f:61)."""
    t = C.c_double(tal)
    mm, d, f, e = C.c_int(m), C.c_double(dt), C.c_double(tf), C.c_double(de)
    N.load().hwhm_(C.byref(mm), C.byref(d), C.byref(f), C.byref(t), C.byref(e),
                   C.c_void_p(u.ctypes.data), C.c_void_p(v.ctypes.data))
    return t.value


def spectrumtd(tpwind, m, dt, tf, wp, de, u, v):
    """SPECTRUMTD in place on float64 arrays u, v (prints the spectrum
    table); returns DE as the reference leaves it (negative -> 0)."""
    e = C.c_double(de)
    mm, d, f, w = C.c_int(m), C.c_double(dt), C.c_double(tf), C.c_double(wp)
    b = tpwind.encode()
    N.load().spectrumtd_(b, C.byref(mm), C.byref(d), C.byref(f), C.byref(w), C.byref(e),
                         C.c_void_p(u.ctypes.data), C.c_void_p(v.ctypes.data), len(b))
    return e.value
