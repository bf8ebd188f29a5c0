"""Python mirror of eSPec's FFT propagator subroutines, called through the
Fortran ABI of libespecgpu.so (`pspofft_`, `psodfft_`).

`pspofft` and `psodfft` take the arguments of PSPOFFT (pspofft.f:1-3) and
PSODFFT (psodfft.f:1-3) by name, with the same meaning, and update the same
arrays in place: U1/V1 (and U2/V2), TC and the LNZVC columns MPR/MPI
(LNZVC is a Fortran-ordered (MXDCT, ncols) array; MPR/MPI are 1-based).
They return INFO: 0, 1 for a drift beyond TOL percent, 2 for a case the GPU
path does not run or a device error (the reason goes to standard error).  The partial
auto-correlation table goes to standard output when PRTCRL is '.YES' or
'.PARTIAL', as the reference prints it.
"""
import ctypes as C

import numpy as np

from . import _native as N


def _arr(a):
    if (not isinstance(a, np.ndarray) or a.dtype != np.float64
            or not (a.flags.c_contiguous or a.flags.f_contiguous)):
        raise TypeError("arrays updated in place must be contiguous float64 numpy arrays")
    return C.c_void_p(a.ctypes.data)


def _common(absorb, dim, prtcrl, tpabsor, lc, mp, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_, sh,
            sm):
    keep = dict(
        absorb=C.c_int(1 if absorb else 0), lc=C.c_int(lc), mp=C.c_int(mp), mpi=C.c_int(mpi),
        mpr=C.c_int(mpr), mxdct=C.c_int(mxdct), n=C.c_int(n), dt=C.c_double(dt),
        ti=C.c_double(ti), tf=C.c_double(tf), tol=C.c_double(tol),
        np=np.ascontiguousarray(np_, dtype=np.int32), sh=N.f64(sh), sm=N.f64(sm),
        shm=np.zeros(3), dummy=np.zeros(1),
        dim=dim.encode(), prtcrl=prtcrl.encode(), tpabsor=tpabsor.encode())
    return keep


def pspofft(*, absorb, dim, prtcrl, tpabsor, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_, sh,
            sm, u1, v1, tc, vpot, vabc, lnzvc, mp=0):
    """PSPOFFT: split-operator propagation of U1 + i V1 from TI to TF (fs)."""
    k = _common(absorb, dim, prtcrl, tpabsor, lc, mp, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_,
                sh, sm)
    info = C.c_int(0)
    vp = N.f64(vpot)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    N.load().pspofft_(
        C.byref(k["absorb"]), k["dim"], k["prtcrl"], k["tpabsor"], C.byref(info), C.byref(k["lc"]),
        C.byref(k["mp"]), C.byref(k["mpi"]), C.byref(k["mpr"]), C.byref(k["mxdct"]),
        C.byref(k["n"]), C.byref(k["dt"]), C.byref(k["ti"]), C.byref(k["tf"]), C.byref(k["tol"]),
        N.ptr(k["np"]), N.ptr(k["shm"]), N.ptr(k["sh"]), N.ptr(k["sm"]), _arr(u1), _arr(v1),
        N.ptr(k["dummy"]), N.ptr(k["dummy"]), _arr(tc), N.ptr(vp), N.ptr(va), _arr(lnzvc),
        N.ptr(k["dummy"]), N.ptr(k["dummy"]), N.ptr(k["dummy"]),
        len(k["dim"]), len(k["prtcrl"]), len(k["tpabsor"]))
    return info.value


def psodfft(*, absorb, dim, prtcrl, tpabsor, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_, sh,
            sm, u1, u2, v1, v2, tc, vpot, vabc, lnzvc, mp=0):
    """PSODFFT: second-order-differences propagation; on return U2 + i V2 is
    psi(TF) and U1 + i V1 is psi(TF - dt)."""
    k = _common(absorb, dim, prtcrl, tpabsor, lc, mp, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_,
                sh, sm)
    info = C.c_int(0)
    vp = N.f64(vpot)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    N.load().psodfft_(
        C.byref(k["absorb"]), k["dim"], k["prtcrl"], k["tpabsor"], C.byref(info), C.byref(k["lc"]),
        C.byref(k["mp"]), C.byref(k["mpi"]), C.byref(k["mpr"]), C.byref(k["mxdct"]),
        C.byref(k["n"]), C.byref(k["dt"]), C.byref(k["ti"]), C.byref(k["tf"]), C.byref(k["tol"]),
        N.ptr(k["np"]), N.ptr(k["shm"]), N.ptr(k["sh"]), N.ptr(k["sm"]), _arr(u1), _arr(u2),
        _arr(v1), _arr(v2), N.ptr(k["dummy"]), N.ptr(k["dummy"]), _arr(tc), N.ptr(vp), N.ptr(va),
        N.ptr(k["dummy"]), N.ptr(k["dummy"]), N.ptr(k["dummy"]), _arr(lnzvc),
        len(k["dim"]), len(k["prtcrl"]), len(k["tpabsor"]))
    return info.value


def plnz(*, absorb, change, dim, prtcrl, tpabsor, lc, lmtreort, mp, mpi, mpr, mxdct, n, dt,
         ti, tf, tol, np_, shm, vpot, vabc, u, v, lnzvc, abstol=1e-6):
    """PLNZ: short-iterative-Lanczos propagation of U + i V (1D/2D/3D grid,
    flattened x fastest).  Returns (INFO, MP after the call: LNZ lowers MP to
    LMTREORT when *CHANGE is on, lnz.f:64-72)."""
    info = C.c_int(0)
    mp_c = C.c_int(mp)
    npa = np.array(list(np_) + [1] * (3 - len(np_)), dtype=np.int32)
    shma = N.f64(list(shm) + [0.0] * (3 - len(shm)))
    vp = N.f64(vpot)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    sc = dict(absorb=C.c_int(1 if absorb else 0), change=C.c_int(1 if change else 0),
              lc=C.c_int(lc), lmt=C.c_int(lmtreort), mpi=C.c_int(mpi), mpr=C.c_int(mpr),
              mxdct=C.c_int(mxdct), n=C.c_int(n), abstol=C.c_double(abstol), dt=C.c_double(dt),
              ti=C.c_double(ti), tf=C.c_double(tf), tol=C.c_double(tol))
    scratch = np.zeros(max(n, 1))
    iwork = np.zeros(16, dtype=np.int32)
    b = {k: v.encode() for k, v in dict(dim=dim, prtcrl=prtcrl, tpabsor=tpabsor).items()}
    N.load().plnz_(
        C.byref(sc["absorb"]), C.byref(sc["change"]), b["dim"], b["prtcrl"], b["tpabsor"],
        C.byref(info), C.byref(sc["lc"]), C.byref(sc["lmt"]), C.byref(mp_c), C.byref(sc["mpi"]),
        C.byref(sc["mpr"]), C.byref(sc["mxdct"]), C.byref(sc["n"]), C.byref(sc["abstol"]),
        C.byref(sc["dt"]), C.byref(sc["ti"]), C.byref(sc["tf"]), C.byref(sc["tol"]), N.ptr(npa),
        N.ptr(iwork), N.ptr(shma), N.ptr(vp), N.ptr(va), _arr(u), _arr(v), N.ptr(scratch),
        N.ptr(scratch), N.ptr(scratch), N.ptr(scratch), N.ptr(scratch), N.ptr(scratch),
        N.ptr(scratch), _arr(lnzvc), len(b["dim"]), len(b["prtcrl"]), len(b["tpabsor"]))
    return info.value, mp_c.value


def psod(*, absorb, dim, prtcrl, tpabsor, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_, shm,
         vpot, vabc, u1, v1, u2, v2, lnzvc, mp=0):
    """PSOD: second-order differences with the finite-difference Hamiltonian
    (1D/2D/3D grid, flattened x fastest); on return U2 + i V2 is psi(TF) and
    U1 + i V1 is psi(TF - dt).  Returns INFO."""
    info = C.c_int(0)
    npa = np.array(list(np_) + [1] * (3 - len(np_)), dtype=np.int32)
    shma = N.f64(list(shm) + [0.0] * (3 - len(shm)))
    vp = N.f64(vpot)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    sc = dict(absorb=C.c_int(1 if absorb else 0), lc=C.c_int(lc), mp=C.c_int(mp),
              mpi=C.c_int(mpi), mpr=C.c_int(mpr), mxdct=C.c_int(mxdct), n=C.c_int(n),
              dt=C.c_double(dt), ti=C.c_double(ti), tf=C.c_double(tf), tol=C.c_double(tol))
    scratch = np.zeros(max(n, 1))
    xi = np.zeros(3)
    b = {k: v.encode() for k, v in dict(dim=dim, prtcrl=prtcrl, tpabsor=tpabsor).items()}
    N.load().psod_(
        C.byref(sc["absorb"]), b["dim"], b["prtcrl"], b["tpabsor"], C.byref(info),
        C.byref(sc["lc"]), C.byref(sc["mp"]), C.byref(sc["mpi"]), C.byref(sc["mpr"]),
        C.byref(sc["mxdct"]), C.byref(sc["n"]), C.byref(sc["dt"]), C.byref(sc["ti"]),
        C.byref(sc["tf"]), C.byref(sc["tol"]), N.ptr(npa), N.ptr(shma), _arr(u1), _arr(u2),
        _arr(v1), _arr(v2), N.ptr(xi), N.ptr(xi), N.ptr(vp), N.ptr(va), N.ptr(scratch),
        N.ptr(scratch), _arr(lnzvc), len(b["dim"]), len(b["prtcrl"]), len(b["tpabsor"]))
    return info.value


def ppsod(*, absorb, dim, efc, prtcrl, tpabsor, lc, mpi, mpr, mxdct, n, dt, ti, tf, tol, np_,
          shm, e0, tp, omg, dm, vpot, vabc, u1, v1, u2, v2, lnzvc, t0=0.0, td=0.0, sni=0.0, kl=0,
          npr=0, kp=1, nispg=1):
    """PPSOD: PSOD with the laser pulse efc ('.GAUS', '.GGAUS', '.SIN2',
    '.NONE') and the dipole function dm; the projection vectors are the
    columns kp..kp+npr-1 (0-based) of lnzvc.  On return U2 + i V2 is psi(TF),
    U1 + i V1 is psi(TF - dt) and vpot holds VP - DM EF of the last step.
    Returns INFO."""
    info = C.c_int(0)
    npa = np.array(list(np_) + [1] * (3 - len(np_)), dtype=np.int32)
    shma = N.f64(list(shm) + [0.0] * (3 - len(shm)))
    dma = N.f64(dm)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    ints = {k: C.c_int(v) for k, v in dict(
        absorb=1 if absorb else 0, off=0, lc=lc, mp=0, mpi=mpi, mpr=mpr, mxdct=mxdct, n=n,
        nshot=10, npr=npr, kp=kp, nispg=nispg, kl=kl).items()}
    dbl = {k: C.c_double(v) for k, v in dict(
        e0=e0, t0=t0, td=td, tp=tp, omg=omg, sni=sni, dt=dt, ti=ti, tf=tf, tol=tol).items()}
    z3 = np.zeros(3)
    scratch = np.zeros(max(n, 1))
    rng = np.zeros(36)
    b = {k: v.encode() for k, v in dict(dim=dim, efc=efc, prtcrl=prtcrl, tpabsor=tpabsor).items()}
    r = C.byref
    N.load().ppsod_(
        r(ints["absorb"]), r(ints["off"]), r(ints["off"]), r(ints["off"]), b["dim"], b["efc"],
        b["prtcrl"], b["tpabsor"], r(info), r(ints["lc"]), r(ints["mp"]), r(ints["mpi"]),
        r(ints["mpr"]), r(ints["mxdct"]), r(ints["n"]), r(ints["nshot"]), r(ints["npr"]),
        r(ints["kp"]), r(ints["nispg"]), r(dbl["e0"]), r(dbl["t0"]), r(dbl["td"]), r(dbl["tp"]),
        r(dbl["omg"]), r(dbl["sni"]), r(ints["kl"]), r(dbl["dt"]), r(dbl["ti"]), r(dbl["tf"]),
        r(dbl["tol"]), N.ptr(npa), N.ptr(npa), N.ptr(z3), N.ptr(shma), _arr(u1), _arr(u2),
        _arr(v1), _arr(v2), N.ptr(z3), N.ptr(z3), N.ptr(z3), N.ptr(dma), _arr(vpot), N.ptr(va),
        N.ptr(scratch), N.ptr(z3), _arr(lnzvc), r(ints["off"]), r(ints["off"]), N.ptr(rng),
        r(ints["off"]), len(b["dim"]), len(b["efc"]), len(b["prtcrl"]), len(b["tpabsor"]))
    return info.value


def pplnz(*, absorb, change, dim, efc, prtcrl, tpabsor, lc, lmtreort, mp, mpi, mpr, mxdct, n,
          dt, ti, tf, tol, np_, shm, e0, tp, omg, dm, vpot, vabc, u, v, lnzvc, t0=0.0, td=0.0,
          sni=0.0, kl=0, npr=0, kp=1, abstol=1e-6):
    """PPLNZ: PLNZ with the laser pulse efc and the dipole function dm; the
    projection vectors are the columns kp..kp+npr-2 (0-based) of lnzvc.  On
    return U + i V is psi(TF) and vpot holds VP - DM EF of the last step.
    Returns (INFO, MP after the call)."""
    info = C.c_int(0)
    mp_c = C.c_int(mp)
    npa = np.array(list(np_) + [1] * (3 - len(np_)), dtype=np.int32)
    shma = N.f64(list(shm) + [0.0] * (3 - len(shm)))
    dma = N.f64(dm)
    va = N.f64(vabc) if vabc is not None else np.zeros(n)
    ints = {k: C.c_int(v) for k, v in dict(
        absorb=1 if absorb else 0, change=1 if change else 0, off=0, lc=lc, lmt=lmtreort,
        mpi=mpi, mpr=mpr, mxdct=mxdct, n=n, nshot=10, kl=kl, npr=npr, kp=kp).items()}
    dbl = {k: C.c_double(v) for k, v in dict(
        abstol=abstol, dt=dt, ti=ti, tf=tf, tol=tol, e0=e0, t0=t0, td=td, tp=tp, omg=omg,
        sni=sni).items()}
    z3 = np.zeros(3)
    scratch = np.zeros(max(n, 1))
    iwork = np.zeros(16, dtype=np.int32)
    b = {k: v.encode() for k, v in dict(dim=dim, efc=efc, prtcrl=prtcrl, tpabsor=tpabsor).items()}
    r = C.byref
    N.load().pplnz_(
        r(ints["absorb"]), r(ints["change"]), r(ints["off"]), r(ints["off"]), r(ints["off"]),
        b["dim"], b["efc"], b["prtcrl"], b["tpabsor"], r(info), r(ints["lc"]), r(ints["lmt"]),
        r(mp_c), r(ints["mpi"]), r(ints["mpr"]), r(ints["mxdct"]), r(ints["n"]), r(ints["nshot"]),
        r(ints["kl"]), r(ints["npr"]), r(ints["kp"]), r(dbl["abstol"]), r(dbl["dt"]),
        r(dbl["ti"]), r(dbl["tf"]), r(dbl["tol"]), r(dbl["e0"]), r(dbl["t0"]), r(dbl["td"]),
        r(dbl["tp"]), r(dbl["omg"]), r(dbl["sni"]), N.ptr(npa), N.ptr(npa), N.ptr(iwork),
        N.ptr(z3), N.ptr(shma), _arr(vpot), N.ptr(va), _arr(u), _arr(v), N.ptr(z3), N.ptr(z3),
        N.ptr(z3), N.ptr(dma), N.ptr(scratch), N.ptr(scratch), N.ptr(scratch), N.ptr(scratch),
        N.ptr(z3), _arr(lnzvc), len(b["dim"]), len(b["efc"]), len(b["prtcrl"]),
        len(b["tpabsor"]))
    return info.value, mp_c.value


def format_crl_row(t, e, cr, ci, ct, fnt):
    """One row of the partial auto-correlation table (FORMAT 1021, pspofft.f:148)."""
    buf = C.create_string_buffer(256)
    n = N.load().espec_format_crl_row(t, e, cr, ci, ct, fnt, buf, 256)
    N.check(0 if n > 0 else n, "espec_format_crl_row")
    return buf.value.decode()
