"""Initial-state eigensolver on the GPU (eSPec's LANCZSG, lanczsc.f:56-120,
with locking and the true residual), batched over potentials, FP64.

Device tensors (torch) carry the data: `morse2d_potentials` builds the 2D
coupled-Morse family on the grid, `lcg_start` the reference's cold-start
vectors (rans.f), `solve` runs the restarted Lanczos and returns
eigenvalues, eigenvectors, residuals and the H*v count per state.
"""
import ctypes as C

import numpy as np

from . import _native as N

RE1, RE2 = 1.4, 1.8  # equilibrium positions of the two Morse modes (bohr)


class Grid2D:
    """np = (nx, ny) points on [xi, xf] x [yi, yf] (bohr), masses m1, m2 (m_e)."""

    def __init__(self, np_=(128, 128), box=(0.6, 3.6, 0.9, 3.9), masses=(918.0, 1500.0)):
        self.np = [int(np_[0]), int(np_[1])]
        self.box = [float(b) for b in box]
        self.n = self.np[0] * self.np[1]
        hx = (self.box[1] - self.box[0]) / (self.np[0] - 1)
        hy = (self.box[3] - self.box[2]) / (self.np[1] - 1)
        self.sh = [hx, hy]
        # SHM = 1/(24 m h^2), multiplied left to right as espec.f:819
        self.shm = [1.0 / (((24.0 * masses[0]) * hx) * hx), 1.0 / (((24.0 * masses[1]) * hy) * hy)]


def _stream(t, stream):
    import torch

    return stream if stream is not None else torch.cuda.current_stream(t.device).cuda_stream


def morse2d_potentials(grid, params):
    """params: torch float64 CUDA tensor [nprob, 5] = (De1, a1, De2, a2, lambda)."""
    import torch

    params = params.contiguous()
    nprob = params.shape[0]
    out = torch.empty((nprob, grid.n), dtype=torch.float64, device=params.device)
    npa = (C.c_int * 2)(*grid.np)
    b = grid.box
    N.check(N.load().espec_eig_morse2d(nprob, params.data_ptr(), npa, b[0], b[1], b[2], b[3], RE1,
                                       RE2, out.data_ptr(), _stream(params, None)),
            "espec_eig_morse2d")
    return out


def lcg_start(n, nstates, device):
    import torch

    out = torch.empty((nstates, n), dtype=torch.float64, device=device)
    N.check(N.load().espec_eig_lcg_start(out.data_ptr(), n, nstates, _stream(out, None)),
            "espec_eig_lcg_start")
    return out


def solve(grid, vpot, start, nstates=4, m=40, tol=1e-9, maxrest=200, stream=None):
    """vpot [nprob, n], start [nprob, nstates, n] (float64 CUDA tensors).
    Returns dict(eval [nprob, nstates], vec [nprob, nstates, n], resid, matvecs)."""
    import torch

    vpot = vpot.contiguous()
    start = start.contiguous()
    nprob = vpot.shape[0]
    dev = vpot.device
    vec = torch.empty((nprob, nstates, grid.n), dtype=torch.float64, device=dev)
    ev = torch.empty((nprob, nstates), dtype=torch.float64, device=dev)
    res = torch.empty_like(ev)
    mv = torch.empty((nprob, nstates), dtype=torch.int32, device=dev)
    wl = torch.empty((nprob, m, grid.n), dtype=torch.float64, device=dev)
    wv = torch.empty((nprob, grid.n), dtype=torch.float64, device=dev)
    npa = (C.c_int * 2)(*grid.np)
    shm = (C.c_double * 2)(*grid.shm)
    rc = N.load().espec_eig_solve_dev(nprob, npa, shm, vpot.data_ptr(), start.data_ptr(), nstates,
                                      m, tol, maxrest, vec.data_ptr(), ev.data_ptr(),
                                      res.data_ptr(), mv.data_ptr(), wl.data_ptr(), wv.data_ptr(),
                                      _stream(vpot, stream))
    N.check(rc, "espec_eig_solve_dev")
    return dict(eval=ev, vec=vec, resid=res, matvecs=mv)
