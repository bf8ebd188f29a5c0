"""Host-side mirror of eSPec's split-operator propagator for batched scans.

`SpoBatch` propagates many independent 1D packets with the split-operator
FFT method of PSPOFFT/PSPOFFTAUX (pspofft.f:72-145, spofft.f:64-200) in one
launch on the GPU.  Units follow the reference: dt in fs, grid step in bohr,
mass in electron masses, potentials in hartree.  Each packet's C(t) is
recorded every step (LC = 1); `c` has nsteps+1 samples with c[0] = C(TI).
"""
import ctypes as C

import numpy as np

from . import _native as N


class SpoBatch:
    method = N.SPO

    def __init__(self, npts, sh, sm, dt_fs, precision="fp64", absorb=N.ABS_NONE, quirks=0):
        lib = N.load()
        self.npts = np.ascontiguousarray(npts, dtype=np.int32)
        self.npk = int(self.npts.size)
        self.off = np.concatenate([[0], np.cumsum(self.npts)]).astype(np.int64)
        self.total = int(self.off[-1])
        self.sh = N.f64(sh)
        self.sm = N.f64(sm)
        self.dt_fs = float(dt_fs)
        self.precision = {"fp64": N.FP64, "mixed": N.MIXED}[precision]
        self.absorb = absorb
        self._h = C.c_void_p()
        rc = lib.espec_prop_create(C.byref(self._h), self.npk,
                                   self.npts.ctypes.data_as(C.POINTER(C.c_int)),
                                   self.sh.ctypes.data_as(C.POINTER(C.c_double)),
                                   self.sm.ctypes.data_as(C.POINTER(C.c_double)),
                                   self.dt_fs, self.method, self.precision, absorb, quirks)
        N.check(rc, "espec_prop_create")
        self.nsteps = None

    def set_launch(self, mode):
        """"persistent" (one kernel over all packet sizes, items claimed
        longest first) or "classes" (one kernel per size class); before load."""
        m = {"classes": N.LAUNCH_CLASSES, "persistent": N.LAUNCH_PERSISTENT}[mode]
        N.check(N.load().espec_spo_set_launch(self._h, m), "espec_spo_set_launch")

    def set_item_cost(self, npts, cost):
        """Relative cost of one persistent item of packets of size npts."""
        N.check(N.load().espec_spo_set_item_cost(self._h, int(npts), float(cost)),
                "espec_spo_set_item_cost")

    def set_variant(self, npts, variant):
        """Choose the kernel variant of one packet size (before load); selects
        the per-class launch."""
        N.check(N.load().espec_spo_set_variant(self._h, int(npts), int(variant)),
                "espec_spo_set_variant")

    def load(self, vpot, psi, vabc=None, stream=None, asynchronous=False):
        """vpot, psi (complex or real), vabc: host numpy arrays (concatenated),
        or device tensors (torch float64) with psi given as (re, im).  With
        asynchronous=True, host (re, im) arrays must be page-locked float64
        arrays that stay untouched until the stream has passed the copies."""
        lib = N.load()
        if isinstance(psi, tuple) and isinstance(psi[0], np.ndarray):  # host (re, im)
            self._keep = [N.f64(vpot), N.f64(psi[0]), N.f64(psi[1]),
                          None if vabc is None else N.f64(vabc)]
            v, re, im, ab = self._keep
            rc = lib.espec_spo_load(self._h, N.ptr(v), N.ptr(ab), N.ptr(re), N.ptr(im),
                                    N.MEM_HOST_ASYNC if asynchronous else N.MEM_HOST, stream)
        elif isinstance(psi, tuple):  # device (re, im)
            re, im = psi
            rc = lib.espec_spo_load(self._h, N.ptr(vpot), N.ptr(vabc), N.ptr(re), N.ptr(im),
                                    N.MEM_DEVICE, stream)
        else:
            psi = np.asarray(psi)
            self._keep = [N.f64(vpot), N.f64(psi.real), N.f64(np.imag(psi)),
                          None if vabc is None else N.f64(vabc)]
            v, re, im, ab = self._keep
            rc = lib.espec_spo_load(self._h, N.ptr(v), N.ptr(ab), N.ptr(re), N.ptr(im),
                                    N.MEM_HOST, stream)
        N.check(rc, "espec_spo_load")

    def run(self, nsteps, stream=None):
        N.check(N.load().espec_spo_run(self._h, int(nsteps), stream), "espec_spo_run")
        self.nsteps = int(nsteps)

    def advance(self, nsteps, stream=None):
        """nsteps more steps from the current state; C(t) samples 1..nsteps of
        this call (sample 0 is not written) -- how PSPOFFT's printed rows
        split a run (pspofft.f:125-144)."""
        N.check(N.load().espec_prop_continue(self._h, int(nsteps), stream), "espec_prop_continue")
        self.nsteps = int(nsteps)

    def energies(self, stream=None):
        """(E, norm) of every packet's current state: EFFT4 (eigenergfft.f:58-100)
        in hartree and sum |psi|^2, FP64 on the GPU."""
        e = np.zeros(self.npk)
        nr = np.zeros(self.npk)
        N.check(N.load().espec_prop_energies(self._h, N.ptr(e), N.ptr(nr), stream),
                "espec_prop_energies")
        return e, nr

    def results(self, stream=None):
        """(C(t) [npk, nsteps+1] complex, psi(TF) concatenated complex), host."""
        ns = self.nsteps
        cr = np.zeros(self.npk * (ns + 1))
        ci = np.zeros_like(cr)
        pr = np.zeros(self.total)
        pi = np.zeros(self.total)
        rc = N.load().espec_spo_results(self._h, N.ptr(cr), N.ptr(ci), N.ptr(pr), N.ptr(pi),
                                        N.MEM_HOST, stream)
        N.check(rc, "espec_spo_results")
        return (cr + 1j * ci).reshape(self.npk, ns + 1), pr + 1j * pi

    def results_into(self, c_re, c_im, psi_re, psi_im, stream=None, asynchronous=False):
        """Copy C(t) ([npk * (nsteps+1)], packet-major) and psi(TF) as separate
        real and imaginary float64 host arrays into the caller's buffers (any
        may be None); returns when the copies are done, or at once with
        asynchronous=True (page-locked buffers; synchronise the stream before
        reading them)."""
        where = N.MEM_HOST_ASYNC if asynchronous else N.MEM_HOST
        N.check(N.load().espec_spo_results(self._h, N.ptr(c_re), N.ptr(c_im), N.ptr(psi_re),
                                           N.ptr(psi_im), where, stream),
                "espec_spo_results")

    def nonfinite(self, stream=None):
        """Packets whose C(t) went NaN/Inf during the last run or segment."""
        n = C.c_int(0)
        N.check(N.load().espec_prop_nonfinite(self._h, C.byref(n), stream), "espec_prop_nonfinite")
        return n.value

    def device_c(self):
        """Device address of C(t) (double2, packet-major)."""
        return N.load().espec_spo_device_c(self._h)

    def close(self):
        if self._h:
            N.load().espec_spo_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SodBatch(SpoBatch):
    """Batched second-order-differences propagation with the FFT kinetic term
    (PSODFFT, psodfft.f:77-206), FP64.  Step 1 is the reference's start-up of
    two half steps; `previous()` returns psi(TF - dt)."""

    method = N.SOD

    def __init__(self, npts, sh, sm, dt_fs, absorb=N.ABS_NONE, quirks=0):
        super().__init__(npts, sh, sm, dt_fs, precision="fp64", absorb=absorb, quirks=quirks)

    def previous(self, stream=None):
        pr = np.zeros(self.total)
        pi = np.zeros(self.total)
        N.check(N.load().espec_prop_previous(self._h, N.ptr(pr), N.ptr(pi), N.MEM_HOST, stream),
                "espec_prop_previous")
        return pr + 1j * pi


def digt_1d(n, sh, sm):
    """dkeft.f:64-79 kinetic table (FFT order), truncated 2 pi as the reference."""
    twopi = 6.283185307
    dp = twopi / (n * sh)
    tc = np.empty(n)
    p = 0.0
    for i in range(n // 2):
        tc[i] = p * p / (2.0 * sm)
        p = p + dp
    p = -p
    for i in range(n // 2, n):
        tc[i] = p * p / (2.0 * sm)
        p = p + dp
    return tc
