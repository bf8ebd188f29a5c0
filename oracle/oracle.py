"""ctypes binding of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: this module is the checker.  It may be imported by
tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline / reference
legs -- never by the espec_b200 product package.

Each wrapper mirrors one routine of the reference's src/ (cited in
espec_oracle.cpp); arrays are numpy float64, 0-based, x fastest.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

Q_SPO_INPLACE = 1
Q_SIL_INPLACE = 2
Q_DIGT_ND = 4
Q_SOD_SMOOTHW = 8
Q_FFTNT_SP = 16
Q_PSOD_COPY = 32
Q_ALL = 31

ABS_NONE, ABS_VOPTIC, ABS_SMOOTHW = 0, 1, 2
PRT_NONE, PRT_PARTIAL, PRT_YES = 0, 1, 2
ABC_SMOOTHW, ABC_VOPTIC_LINEAR, ABC_VOPTIC_POLIN, ABC_SMRS = 1, 2, 3, 4

SHFS = 2.4188843243e-2   # pspofft.f:76
A0A = 0.5291772083       # espec.f:67
AMU = 1836.152667539     # espec.f:614
FATE = 27.2113834        # spectrumtd.f:38


class Prop(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("np", C.c_int * 3),
        ("dt", C.c_double), ("ti", C.c_double), ("tf", C.c_double),
        ("tol", C.c_double),
        ("sh", C.c_double * 3), ("sm", C.c_double * 3), ("shm", C.c_double * 3),
        ("lc", C.c_int), ("absorb", C.c_int), ("prtcrl", C.c_int),
        ("quirks", C.c_int), ("mp", C.c_int), ("lmtreort", C.c_int),
        ("change", C.c_int),
    ]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        d = C.POINTER(C.c_double)
        i = C.POINTER(C.c_int)
        _lib.orc_do_count.restype = C.c_int
        _lib.orc_do_count.argtypes = [C.c_double] * 3
        _lib.orc_fcorrel.restype = C.c_double
        _lib.orc_ecnorm.restype = C.c_double
        _lib.orc_eigenerg.restype = C.c_double
        _lib.orc_ef.restype = C.c_double
        _lib.orc_ef.argtypes = [C.c_int, C.c_void_p, C.c_double]
        _lib.orc_efft4.restype = C.c_double
        _lib.orc_efft4.argtypes = [C.c_int, i, C.c_double, d, d, d, d]
        _lib.orc_spo_step.argtypes = [C.c_int, i, C.c_double, C.c_double, C.c_double,
                                      d, d, d, C.c_int, C.c_int, d, d]
        _lib.orc_hwhm.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_double, d, d]
        _lib.orc_spectrumtd.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, d, d, d, C.c_int]
        _lib.orc_spo_batch.argtypes = [C.c_int, i, d, d, d, d, d, C.c_double,
                                       C.c_int, C.c_int, d, d, C.c_int]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def do_count(a, b, c):
    return lib().orc_do_count(a, b, c)


def fft(re, im, n, nspan, isn):
    re, im = f64(re).copy(), f64(im).copy()
    lib().orc_fft(_p(re), _p(im), C.c_int(re.size), C.c_int(n), C.c_int(nspan), C.c_int(isn))
    return re, im


def digt(np_, sh, sm, quirks=0):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    sha = f64(list(sh) + [1.0] * (3 - nd))
    sma = f64(list(sm) + [1.0] * (3 - nd))
    n = int(np.prod(np_))
    tc = np.zeros(n)
    b = C.c_double()
    lib().orc_digt(C.c_int(nd), _ip(npa), _p(sha), _p(sma), _p(tc), C.byref(b), C.c_int(quirks))
    return tc, b.value


def au(np_, shm, vpot, u):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    shma = f64(list(shm) + [0.0] * (3 - nd))
    out = np.zeros(int(np.prod(np_)))
    vpot, u = f64(vpot), f64(u)
    lib().orc_au(C.c_int(nd), _ip(npa), _p(shma), _p(vpot), _p(u), _p(out))
    return out


def tridiag_eig(d, e):
    d = f64(d)
    n = d.size
    e = f64(list(e) + [0.0] * (n - len(e)))
    w = np.zeros(n)
    z = np.zeros(n * n)
    rc = lib().orc_tridiag_eig(C.c_int(n), _p(d), _p(e), _p(w), _p(z))
    if rc:
        raise RuntimeError("tridiagonal eigensolver did not converge")
    return w, z.reshape(n, n).T.copy()  # columns = eigenvectors


def efft4(np_, u, v, tc, vpot, b):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    u, v, tc, vpot = f64(u), f64(v), f64(tc), f64(vpot)
    return lib().orc_efft4(nd, _ip(npa), b, _p(u), _p(v), _p(tc), _p(vpot))


def eigenerg(np_, shm, vpot, u):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    shma = f64(list(shm) + [0.0] * (3 - nd))
    u, vpot = f64(u), f64(vpot)
    return lib().orc_eigenerg(C.c_int(nd), _ip(npa), _p(shma), _p(vpot), _p(u))


def make_prop(np_, dt, ti, tf, sh, sm, lc=1, tol=1e9, absorb=ABS_NONE,
              prtcrl=PRT_NONE, quirks=0, mp=10, lmtreort=10, change=1, shm=None):
    nd = len(np_)
    p = Prop()
    p.ndim = nd
    for a in range(3):
        p.np[a] = np_[a] if a < nd else 1
        p.sh[a] = sh[a] if a < nd else 1.0
        p.sm[a] = sm[a] if a < nd else 1.0
        if shm is not None:
            p.shm[a] = shm[a] if a < nd else 0.0
        else:
            p.shm[a] = 1.0 / (24.0 * sm[a] * sh[a] * sh[a]) if a < nd else 0.0
    p.dt, p.ti, p.tf, p.tol = dt, ti, tf, tol
    p.lc, p.absorb, p.prtcrl, p.quirks = lc, absorb, prtcrl, quirks
    p.mp, p.lmtreort, p.change = mp, lmtreort, change
    return p


def _run(fn, p, vpot, vabc, arrays, max_c, max_rows):
    n = int(np.prod([p.np[a] for a in range(p.ndim)]))
    vpot = f64(vpot)
    vabc = f64(vabc) if vabc is not None else np.zeros(n)
    cre = np.zeros(max_c)
    cim = np.zeros(max_c)
    rows = np.zeros(6 * max_rows)
    nrows = C.c_int()
    info = C.c_int()
    nc = fn(C.byref(p), _p(vpot), _p(vabc), *[_p(a) for a in arrays], _p(cre), _p(cim),
            C.c_int(max_c), _p(rows), C.c_int(max_rows), C.byref(nrows), C.byref(info))
    if nc < 0:
        raise RuntimeError("oracle propagation stopped (reference STOP condition)")
    nr = min(nrows.value, max_rows)
    return dict(c=cre[:min(nc, max_c)] + 1j * cim[:min(nc, max_c)],
                rows=rows[:6 * nr].reshape(nr, 6), info=info.value, nc=nc)


def _caps(p):
    nsteps = do_count(p.ti + p.dt, p.tf + p.dt, p.dt) + 2
    max_c = nsteps // max(p.lc, 1) + 2
    max_rows = (nsteps + 2) if p.prtcrl == PRT_YES else (max_c + 2 if p.prtcrl else 1)
    return max_c, max_rows


def pspofft(p, vpot, u, v, vabc=None):
    u, v = f64(u).copy(), f64(v).copy()
    r = _run(lib().orc_pspofft, p, vpot, vabc, [u, v], *_caps(p))
    r.update(u=u, v=v)
    return r


def psodfft(p, vpot, u, v, vabc=None):
    u1, v1 = f64(u).copy(), f64(v).copy()
    u2, v2 = np.zeros_like(u1), np.zeros_like(v1)
    r = _run(lib().orc_psodfft, p, vpot, vabc, [u1, v1, u2, v2], *_caps(p))
    r.update(u=u2, v=v2, u_prev=u1, v_prev=v1)
    return r


def psod(p, vpot, u, v, vabc=None):
    u1, v1 = f64(u).copy(), f64(v).copy()
    u2, v2 = np.zeros_like(u1), np.zeros_like(v1)
    r = _run(lib().orc_psod, p, vpot, vabc, [u1, v1, u2, v2], *_caps(p))
    r.update(u=u2, v=v2, u_prev=u1, v_prev=v1)
    return r


def ef(shape, par, t):
    return lib().orc_ef(int(shape), _p(f64(list(par) + [0.0] * (6 - len(par)))), float(t))


def ppsod(p, vp, dm, shape, par, u, v, vabc=None):
    """PPSOD's propagation: C(t) every LC steps, psi(TF), psi(TF - dt)."""
    n = int(np.prod([p.np[a] for a in range(p.ndim)]))
    u1, v1 = f64(u).copy(), f64(v).copy()
    u2, v2 = np.zeros_like(u1), np.zeros_like(v1)
    max_c, _ = _caps(p)
    cre, cim = np.zeros(max_c + 4), np.zeros(max_c + 4)
    vabc = f64(vabc) if vabc is not None else np.zeros(n)
    parr = f64(list(par) + [0.0] * (6 - len(par)))
    nc = lib().orc_ppsod(C.byref(p), _p(f64(vp)), _p(vabc), _p(f64(dm)), int(shape), _p(parr),
                         _p(u1), _p(v1), _p(u2), _p(v2), _p(cre), _p(cim), C.c_int(max_c + 4))
    nc = min(nc, max_c + 4)
    return dict(c=cre[:nc] + 1j * cim[:nc], u=u2, v=v2, u_prev=u1, v_prev=v1, nc=nc)


def ppsod_table(p, vp, dm, shape, par, w, u, v, vabc=None):
    """PPSOD with its printed rows (T, ET, E0, Cr, Ci, |C|^2, |P_k|^2.., FNT),
    the LNZVC C(t) rows, INFO, psi(TF) and psi(TF - dt); w: [npr, n] real."""
    n = int(np.prod([p.np[a] for a in range(p.ndim)]))
    w = f64(w).reshape(-1, n)
    npr = w.shape[0]
    u1, v1 = f64(u).copy(), f64(v).copy()
    u2, v2 = np.zeros_like(u1), np.zeros_like(v1)
    nsteps = do_count(p.ti + p.dt, p.tf + p.dt, p.dt) + 4
    max_c = nsteps // max(p.lc, 1) + 4
    cre, cim = np.zeros(max_c), np.zeros(max_c)
    rows = np.zeros((nsteps + 4) * (7 + npr))
    nrows, info = C.c_int(), C.c_int()
    vabc = f64(vabc) if vabc is not None else np.zeros(n)
    parr = f64(list(par) + [0.0] * (6 - len(par)))
    nc = lib().orc_ppsod_table(C.byref(p), _p(f64(vp)), _p(vabc), _p(f64(dm)), int(shape),
                               _p(parr), npr, _p(np.ascontiguousarray(w) if npr else np.zeros(1)), _p(u1), _p(v1), _p(u2),
                               _p(v2), _p(cre), _p(cim), C.c_int(max_c), _p(rows),
                               C.c_int(nsteps + 4), C.byref(nrows), C.byref(info))
    nr = min(nrows.value, nsteps + 4)
    return dict(c=cre[:nc] + 1j * cim[:nc], rows=rows[:nr * (7 + npr)].reshape(nr, 7 + npr),
                info=info.value, u=u2, v=v2, u_prev=u1, v_prev=v1, nc=nc)


def pplnz(p, vp, dm, shape, par, u, v, vabc=None):
    """PPLNZ's propagation: C(t) every LC steps and psi(TF)."""
    n = int(np.prod([p.np[a] for a in range(p.ndim)]))
    u, v = f64(u).copy(), f64(v).copy()
    max_c, _ = _caps(p)
    cre, cim = np.zeros(max_c + 4), np.zeros(max_c + 4)
    vabc = f64(vabc) if vabc is not None else np.zeros(n)
    parr = f64(list(par) + [0.0] * (6 - len(par)))
    nc = lib().orc_pplnz(C.byref(p), _p(f64(vp)), _p(vabc), _p(f64(dm)), int(shape), _p(parr),
                         _p(u), _p(v), _p(cre), _p(cim), C.c_int(max_c + 4))
    if nc < 0:
        raise RuntimeError("oracle propagation stopped (reference STOP condition)")
    nc = min(nc, max_c + 4)
    return dict(c=cre[:nc] + 1j * cim[:nc], u=u, v=v, nc=nc)


def pplnz_table(p, vp, dm, shape, par, npr, w, u, v, vabc=None):
    """PPLNZ with its printed rows (T, ET, E0, Cr, Ci, CT(1..npr), FNT), the
    LNZVC C(t) rows, INFO and psi(TF); w: [npr - 1, n] real (the printed
    projections)."""
    n = int(np.prod([p.np[a] for a in range(p.ndim)]))
    w = f64(w).reshape(-1, n) if npr > 1 else np.zeros((1, n))
    u, v = f64(u).copy(), f64(v).copy()
    nsteps = do_count(p.ti + p.dt, p.tf + p.dt / 2.0, p.dt) + 4
    max_c = nsteps // max(p.lc, 1) + 4
    cre, cim = np.zeros(max_c), np.zeros(max_c)
    ncol = 6 + max(npr, 0)
    rows = np.zeros((nsteps + 4) * ncol)
    nrows, info = C.c_int(), C.c_int()
    vabc = f64(vabc) if vabc is not None else np.zeros(n)
    parr = f64(list(par) + [0.0] * (6 - len(par)))
    nc = lib().orc_pplnz_table(C.byref(p), _p(f64(vp)), _p(vabc), _p(f64(dm)), int(shape),
                               _p(parr), int(npr), _p(np.ascontiguousarray(w)), _p(u), _p(v),
                               _p(cre), _p(cim), C.c_int(max_c), _p(rows), C.c_int(nsteps + 4),
                               C.byref(nrows), C.byref(info))
    if nc < 0:
        raise RuntimeError("oracle propagation stopped (reference STOP condition)")
    nr = min(nrows.value, nsteps + 4)
    return dict(c=cre[:nc] + 1j * cim[:nc], rows=rows[:nr * ncol].reshape(nr, ncol),
                info=info.value, u=u, v=v, nc=nc)


def plnz(p, vpot, u, v, vabc=None):
    u, v = f64(u).copy(), f64(v).copy()
    r = _run(lib().orc_plnz, p, vpot, vabc, [u, v], *_caps(p))
    r.update(u=u, v=v)
    return r


def spo_step(np_, dt_fs, tc, b, vpot, u, v, vabc=None, absorb=ABS_NONE, quirks=0):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    u, v = f64(u).copy(), f64(v).copy()
    tc, vpot = f64(tc), f64(vpot)
    vabc = f64(vabc) if vabc is not None else np.zeros_like(u)
    lib().orc_spo_step(nd, _ip(npa), b, dt_fs / SHFS, dt_fs / (2 * SHFS), _p(tc), _p(vpot),
                       _p(vabc), absorb, quirks, _p(u), _p(v))
    return u, v


def absorbingbc(np_, kind, al, ar, sh, xi, xf, voi):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    pad = lambda a, z: f64(list(a) + [z] * (3 - len(a)))
    out = np.zeros(int(np.prod(np_)))
    rc = lib().orc_absorbingbc(C.c_int(nd), _ip(npa), C.c_int(kind), _p(pad(al, 0)),
                               _p(pad(ar, 0)), _p(pad(sh, 1)), _p(pad(xi, 0)), _p(pad(xf, 0)),
                               _p(pad(voi, 0)), _p(out))
    if rc:
        raise ValueError("absorber not implemented in the reference for this case")
    return out


def total_correlation(mf, c):
    c = np.asarray(c)
    cre, cim = f64(c.real), f64(c.imag)
    n = 1 << mf
    u, v = np.zeros(n), np.zeros(n)
    lib().orc_total_correlation(C.c_int(mf), _p(cre), _p(cim), _p(u), _p(v))
    return u, v


def hwhm(mf, dtf, tf, tal, de, u, v):
    u, v = f64(u).copy(), f64(v).copy()
    lib().orc_hwhm(mf, dtf, tf, tal, de, _p(u), _p(v))
    return u, v


def fftnt(x, y, itype, quirks=0):
    x, y = f64(x).copy(), f64(y).copy()
    n = x.size
    m = int(round(np.log2(n)))
    lib().orc_fftnt(_p(x), _p(y), C.c_int(n), C.c_int(m), C.c_int(itype), C.c_int(quirks))
    return x, y


def spectrumtd(window_sg, mf, dtf, tf, wp, de, u, v, quirks=0):
    u, v = f64(u).copy(), f64(v).copy()
    en = np.zeros(1 << mf)
    lib().orc_spectrumtd(int(window_sg), mf, dtf, tf, wp, de, _p(u), _p(v), _p(en), quirks)
    return en, u, v


def lcg_start(n, nstates):
    out = np.zeros(n * nstates)
    lib().orc_lcg_start(C.c_int(n), C.c_int(nstates), _p(out))
    return out.reshape(nstates, n)


def eig_lanczsg(np_, shm, vpot, nstates, m, tol, maxrest, start):
    nd = len(np_)
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    shma = f64(list(shm) + [0.0] * (3 - nd))
    n = int(np.prod(np_))
    st = f64(np.asarray(start).reshape(-1))
    ev, vec, res = np.zeros(nstates), np.zeros(nstates * n), np.zeros(nstates)
    mv = np.zeros(nstates, dtype=np.int32)
    rc = lib().orc_eig_lanczsg(C.c_int(nd), _ip(npa), _p(shma), _p(f64(vpot)), C.c_int(nstates),
                               C.c_int(m), C.c_double(tol), C.c_int(maxrest), _p(st), _p(ev),
                               _p(vec), _p(res), mv.ctypes.data_as(C.POINTER(C.c_int)))
    return dict(evals=ev, evecs=vec.reshape(nstates, n), resid=res, matvecs=mv, rc=rc)


def spo_batch(off, sh, sm, vpot, u, v, dt_fs, nsteps, nthreads=1, quirks=0):
    off = np.ascontiguousarray(off, dtype=np.int32)
    npk = off.size - 1
    sh, sm, vpot = f64(sh), f64(sm), f64(vpot)
    u, v = f64(u).copy(), f64(v).copy()
    cre = np.zeros(npk * (nsteps + 1))
    cim = np.zeros(npk * (nsteps + 1))
    lib().orc_spo_batch(npk, _ip(off), _p(sh), _p(sm), _p(vpot), _p(u), _p(v), dt_fs,
                        nsteps, quirks, _p(cre), _p(cim), nthreads)
    c = (cre + 1j * cim).reshape(npk, nsteps + 1)
    return c, u, v


def gvpot(shiftp, potch, np_, xi, sh, cst, sm=None, quirk3d=0):
    """GVPOT (gvpot.f) with POT1D/2D/3D (potfuncs.f): (vpot x fastest, XMIN)."""
    nd = len(np_)
    l = lib()
    l.orc_gvpot.argtypes = [C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                            C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                            C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    npa = np.array(list(np_) + [1] * (3 - nd), dtype=np.int32)
    xia = f64(list(xi) + [0.0] * (3 - nd))
    sha = f64(list(sh) + [0.0] * (3 - nd))
    sma = f64(list(sm) + [1.0] * (3 - len(sm))) if sm is not None else f64([1.0, 1.0, 1.0])
    c = np.zeros(14)
    c[:len(cst)] = cst
    out = np.zeros(int(np.prod(np_)))
    xmin = C.c_double(0.0)
    l.orc_gvpot(int(bool(shiftp)), potch.encode(), nd, _ip(npa), _p(xia), _p(sma), _p(sha),
                _p(c), int(quirk3d), _p(out), C.byref(xmin))
    return out, xmin.value
