"""Analytic potentials on the GPU: POT1D/POT2D/POT3D (potfuncs.f) on the grid
loop of GVPOT (gvpot.f), batched over the packets of a 1D scan.

Constants are those GVPOT receives (after MAKECST): atomic units, up to 14
per potential.  Outputs are CUDA float64 tensors (x fastest).
"""
import numpy as np

from . import _native as N


def pot_kind(potch, ndim):
    """ESPEC_POT_* code of the reference's name POTCH for ndim axes (0: none)."""
    b = potch.encode()
    return int(N.load().espec_pot_kind(b, len(b), int(ndim)))


def _kind(potch, ndim):
    k = pot_kind(potch, ndim) if isinstance(potch, str) else int(potch)
    if not k:
        raise N.EspecError(f"no {ndim}D potential form named {potch!r}")
    return k


def gvpot_1d(npts, xi, sh, potch, cst, shiftp=True, out=None, stream=None):
    """npk packets of a scan in one launch: packet k has npts[k] points at
    xi[k] + i sh[k] and constants cst[k] (up to 14).  Returns (vpot, xmin):
    vpot a CUDA tensor (concatenated), xmin the grid minimum per packet."""
    import torch

    npts = np.ascontiguousarray(npts, dtype=np.int32)
    npk = npts.size
    c = np.zeros((npk, 14))
    cst = np.atleast_2d(np.asarray(cst, dtype=np.float64))
    c[:, :cst.shape[1]] = cst
    if out is None:
        out = torch.empty(int(npts.sum()), dtype=torch.float64, device="cuda")
    xmin = np.zeros(npk)
    xi, sh = N.f64(np.broadcast_to(xi, (npk,))), N.f64(np.broadcast_to(sh, (npk,)))
    rc = N.load().espec_gvpot_1d(npk, N.ptr(npts), N.ptr(xi),
                                 N.ptr(sh), _kind(potch, 1), N.ptr(c), int(bool(shiftp)),
                                 out.data_ptr(), N.ptr(xmin),
                                 stream if stream is not None else
                                 torch.cuda.current_stream().cuda_stream)
    N.check(rc, "espec_gvpot_1d")
    return out, xmin


def gvpot_nd(np_, xi, sh, potch, cst, sm=None, shiftp=True, quirks=0, stream=None):
    """One 2D or 3D grid (x fastest) as a CUDA tensor."""
    import torch

    nd = len(np_)
    npa = np.asarray(list(np_), dtype=np.int32)
    c = np.zeros(14)
    c[:len(cst)] = cst
    out = torch.empty(int(np.prod(np_)), dtype=torch.float64, device="cuda")
    sma = N.f64(list(sm) + [1.0] * (3 - len(sm))) if sm is not None else N.f64([1.0, 1.0, 1.0])
    xia, sha = N.f64(xi), N.f64(sh)
    rc = N.load().espec_gvpot_nd(nd, N.ptr(npa), N.ptr(xia), N.ptr(sha), N.ptr(sma),
                                 _kind(potch, nd), N.ptr(c),
                                 int(bool(shiftp)), int(quirks), out.data_ptr(),
                                 stream if stream is not None else
                                 torch.cuda.current_stream().cuda_stream)
    N.check(rc, "espec_gvpot_nd")
    return out
