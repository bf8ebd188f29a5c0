"""Host-side mirror of eSPec's short-iterative-Lanczos propagator on one grid.

`SilGrid` propagates one packet on a 1D, 2D or 3D grid with the method of
PLNZ/PLNZAUX (plnz.f:71-151, sil.f:70-181): per step two Lanczos chains of
order mp with full reorthogonalisation (lnz.f, reort.f), the finite-difference
Hamiltonian of au1d.f/au2di.f/au3d.f and the Krylov exponential, FP64, on the
GPU.  Arrays are flattened x fastest (the reference's column-major U(N)).
Units: dt in fs, shm = 1/(24 m h^2) per axis (espec.f:819), V in hartree.
"""
import ctypes as C

import numpy as np

from . import _native as N


class SilGrid:
    """Short-iterative-Lanczos propagation (PLNZ, plnz.f:71-151) of one packet
    on a 1D/2D/3D grid with the finite-difference Hamiltonian, FP64; with
    precision="mixed" the Lanczos vectors and H psi are FP32 (dot products,
    coefficients, Krylov exponential and state FP64)."""

    method = N.SIL

    def __init__(self, np_, shm, dt_fs, mp, absorb=N.ABS_NONE, quirks=0, precision="fp64"):
        lib = N.load()
        self.np = [int(x) for x in np_]
        self.ndim = len(self.np)
        self.n = int(np.prod(self.np))
        npa = np.array(self.np + [1] * (3 - self.ndim), dtype=np.int32)
        shma = N.f64(list(shm) + [0.0] * (3 - self.ndim))
        self._h = C.c_void_p()
        rc = lib.espec_grid_create(C.byref(self._h), self.method, self.ndim,
                                   npa.ctypes.data_as(C.POINTER(C.c_int)),
                                   shma.ctypes.data_as(C.POINTER(C.c_double)), float(dt_fs),
                                   int(mp), {"fp64": N.FP64, "mixed": N.MIXED}[precision],
                                   absorb, quirks)
        N.check(rc, "espec_grid_create")
        self.nsteps = None

    def load(self, vpot, psi, vabc=None, stream=None):
        psi = np.asarray(psi)
        self._keep = [N.f64(np.ravel(vpot, order="F") if np.ndim(vpot) > 1 else vpot),
                      N.f64(np.real(psi).ravel(order="F") if psi.ndim > 1 else np.real(psi)),
                      N.f64(np.imag(psi).ravel(order="F") if psi.ndim > 1 else np.imag(psi)),
                      None if vabc is None else N.f64(np.ravel(vabc, order="F"))]
        v, re, im, ab = self._keep
        rc = N.load().espec_grid_load(self._h, N.ptr(v), N.ptr(ab), N.ptr(re), N.ptr(im),
                                      N.MEM_HOST, stream)
        N.check(rc, "espec_grid_load")

    def run(self, nsteps, stream=None):
        N.check(N.load().espec_grid_run(self._h, int(nsteps), stream), "espec_grid_run")
        self.nsteps = int(nsteps)

    def advance(self, nsteps, stream=None):
        N.check(N.load().espec_grid_continue(self._h, int(nsteps), stream), "espec_grid_continue")
        self.nsteps = int(nsteps)

    def results(self, stream=None):
        """(C(t) complex [nsteps+1], psi complex [n] flattened x fastest)."""
        ns = self.nsteps
        cr, ci = np.zeros(ns + 1), np.zeros(ns + 1)
        pr, pi = np.zeros(self.n), np.zeros(self.n)
        rc = N.load().espec_grid_results(self._h, N.ptr(cr), N.ptr(ci), N.ptr(pr), N.ptr(pi),
                                         N.MEM_HOST, stream)
        N.check(rc, "espec_grid_results")
        return cr + 1j * ci, pr + 1j * pi

    def energies(self, stream=None):
        """(<u|H u> + <v|H v>, |u|^2 + |v|^2) of the current state (eigenerg.f)."""
        e, nr = C.c_double(), C.c_double()
        N.check(N.load().espec_grid_energies(self._h, C.byref(e), C.byref(nr), stream),
                "espec_grid_energies")
        return e.value, nr.value

    def set_ctas(self, nctas):
        """CTAs of the cooperative launches (0: the plan's maximum)."""
        N.check(N.load().espec_grid_set_ctas(self._h, int(nctas)), "espec_grid_set_ctas")

    def set_pulse(self, dm, ef):
        """A laser pulse (chpot.f): V - dm * ef[j] in PSODAUX call j of a PSOD
        plan (PPSOD; ef from ppsod_field) or in the step landing at step j of a
        SIL plan (PPLNZ; ef from pplnz_field)."""
        self._pulse = (N.f64(np.ravel(dm, order="F")), N.f64(ef))
        N.check(N.load().espec_grid_set_pulse(self._h, N.ptr(self._pulse[0]),
                                              N.ptr(self._pulse[1]), len(self._pulse[1]),
                                              N.MEM_HOST), "espec_grid_set_pulse")

    def energies_at(self, ef, stream=None):
        """(<u|H u> + <v|H v>, norm) with the potential V - dm * ef."""
        e, nr = C.c_double(), C.c_double()
        N.check(N.load().espec_grid_energies_at(self._h, float(ef), C.byref(e), C.byref(nr),
                                                stream), "espec_grid_energies_at")
        return e.value, nr.value

    def close(self):
        if self._h:
            N.load().espec_grid_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PsodGrid(SilGrid):
    """Second-order differences with the finite-difference Hamiltonian (PSOD,
    psod.f:64-205) of one packet on a 1D/2D/3D grid, FP64; `previous()` is
    psi(TF - dt)."""

    method = N.PSOD

    def __init__(self, np_, shm, dt_fs, absorb=N.ABS_NONE, quirks=0):
        super().__init__(np_, shm, dt_fs, 0, absorb=absorb, quirks=quirks)

    def previous(self, stream=None):
        pr, pi = np.zeros(self.n), np.zeros(self.n)
        N.check(N.load().espec_grid_previous(self._h, N.ptr(pr), N.ptr(pi), N.MEM_HOST, stream),
                "espec_grid_previous")
        return pr + 1j * pi

def pulse_field(shape, par, t):
    """E(t) of ef.f for shape N.PULSE_* and par = (E0, TP, OMG, T0 or TD, SNI[, KL])."""
    p = N.f64(list(par) + [0.0] * (6 - len(par)))
    return N.load().espec_pulse_field(int(shape), N.ptr(p), float(t))


def ppsod_field(shape, par, ti, tf, dt):
    """The field of every PSODAUX call of a PPSOD run (start-up calls first);
    the run has len(result) - 1 steps."""
    p = N.f64(list(par) + [0.0] * (6 - len(par)))
    cap = int(round((tf - ti) / dt)) + 8
    ef = np.zeros(cap)
    k = N.load().espec_ppsod_field(int(shape), N.ptr(p), float(ti), float(tf), float(dt),
                                   N.ptr(ef), cap)
    N.check(0 if k > 0 else int(k), "espec_ppsod_field")
    return ef[:k]


def pplnz_field(shape, par, ti, tf, dt):
    """The field of every step of a PPLNZ run (ef[0] at TI); the run has
    len(result) - 1 steps."""
    p = N.f64(list(par) + [0.0] * (6 - len(par)))
    cap = int(round((tf - ti) / dt)) + 8
    ef = np.zeros(cap)
    k = N.load().espec_pplnz_field(int(shape), N.ptr(p), float(ti), float(tf), float(dt),
                                   N.ptr(ef), cap)
    N.check(0 if k > 0 else int(k), "espec_pplnz_field")
    return ef[:k]


class SpoGrid:
    """Split-operator propagation (PSPOFFT/PSPOFFTAUX, pspofft.f:72-145,
    spofft.f:64-200) of one packet on a 2D or 3D grid, FP64 or mixed, on the
    GPU.  np: points per axis (32..512, powers of two), sh/sm per axis (bohr,
    electron masses), arrays flattened x fastest."""

    method = N.SPO

    def __init__(self, np_, sh, sm, dt_fs, precision="fp64", absorb=N.ABS_NONE, quirks=0):
        lib = N.load()
        self.np = [int(x) for x in np_]
        self.n = int(np.prod(self.np))
        npa = np.array(self.np, dtype=np.int32)
        sha, sma = N.f64(sh), N.f64(sm)
        self._h = C.c_void_p()
        rc = lib.espec_spond_create_method(C.byref(self._h), self.method, len(self.np),
                                           npa.ctypes.data_as(C.POINTER(C.c_int)),
                                           sha.ctypes.data_as(C.POINTER(C.c_double)),
                                           sma.ctypes.data_as(C.POINTER(C.c_double)),
                                           float(dt_fs),
                                           {"fp64": N.FP64, "mixed": N.MIXED}[precision], absorb,
                                           quirks)
        N.check(rc, "espec_spond_create_method")
        self.nsteps = None

    def load(self, vpot, psi, vabc=None, stream=None):
        psi = np.asarray(psi)
        self._keep = [N.f64(vpot), N.f64(np.real(psi)), N.f64(np.imag(psi)),
                      None if vabc is None else N.f64(vabc)]
        v, re, im, ab = self._keep
        N.check(N.load().espec_spond_load(self._h, N.ptr(v), N.ptr(ab), N.ptr(re), N.ptr(im),
                                          N.MEM_HOST, stream), "espec_spond_load")

    def run(self, nsteps, stream=None):
        N.check(N.load().espec_spond_run(self._h, int(nsteps), stream), "espec_spond_run")
        self.nsteps = int(nsteps)

    def advance(self, nsteps, stream=None):
        """nsteps more steps from the state of the last run (sample 0 unset)."""
        N.check(N.load().espec_spond_continue(self._h, int(nsteps), stream),
                "espec_spond_continue")
        self.nsteps = int(nsteps)

    def energies(self, stream=None):
        """(EFFT4 energy, sum |psi|^2) of the current state, FP64."""
        e, nr = C.c_double(), C.c_double()
        N.check(N.load().espec_spond_energies(self._h, C.byref(e), C.byref(nr), stream),
                "espec_spond_energies")
        return e.value, nr.value

    def results(self, stream=None):
        ns = self.nsteps
        cr, ci = np.zeros(ns + 1), np.zeros(ns + 1)
        pr, pi = np.zeros(self.n), np.zeros(self.n)
        N.check(N.load().espec_spond_results(self._h, N.ptr(cr), N.ptr(ci), N.ptr(pr), N.ptr(pi),
                                             N.MEM_HOST, stream), "espec_spond_results")
        return cr + 1j * ci, pr + 1j * pi

    def close(self):
        if self._h:
            N.load().espec_spond_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SodGrid(SpoGrid):
    """Second-order-differences propagation with the FFT kinetic term
    (PSODFFT, psodfft.f:77-206) on a 2D or 3D grid, FP64; `previous()` is
    psi(TF - dt)."""

    method = N.SOD

    def __init__(self, np_, sh, sm, dt_fs, absorb=N.ABS_NONE, quirks=0):
        super().__init__(np_, sh, sm, dt_fs, precision="fp64", absorb=absorb, quirks=quirks)

    def previous(self, stream=None):
        pr, pi = np.zeros(self.n), np.zeros(self.n)
        N.check(N.load().espec_spond_previous(self._h, N.ptr(pr), N.ptr(pi), N.MEM_HOST, stream),
                "espec_spond_previous")
        return pr + 1j * pi
