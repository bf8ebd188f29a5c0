"""Learned warm start for the initial-state eigensolver (no counterpart in the
reference, which starts LANCZSG from its LCG vectors, lanczsc.f:56-62).

A small multilayer perceptron maps the five parameters of a 2D coupled-Morse
potential (De1, a1, De2, a2, lambda) to the lowest eigenvectors, written as
coefficients in a fixed product basis phi_i(x) chi_j(y) of the 1D reference
Morse eigenfunctions of each axis.  It is trained on eigenvectors that the
plain eigensolver (espec_b200.eig) itself produces over random parameters,
with the library's own GEMM / activation / loss / Adam kernels (mlp.cu).  Its
proposals are the start vectors of the same solver, which refines them to the
residual tolerance; a problem whose warm-started solve does not converge is
solved again from the cold start (counted).

Everything here runs on the GPU through the C-ABI; torch only holds device
memory.  The host does the bookkeeping of a data set: sampling parameters,
the sign convention of the training eigenvectors, the learning-rate schedule.
"""
import math
from types import SimpleNamespace

import numpy as np

from . import _native as N
from . import eig as EG

# C2-family parameter box (BASELINE's 2D coupled Morse, De/a varied by about
# +-6 % and +-4 %, coupling +-0.01 Eh/bohr^2); inside it the four lowest states
# keep their order (no crossings), so each state is a smooth function of q
PARAM_LO = np.array([0.16, 0.95, 0.11, 1.15, -0.01])
PARAM_HI = np.array([0.18, 1.05, 0.13, 1.25, 0.01])
REF_X = (0.17, 1.0)   # reference Morse of the x basis (De, a), re = 1.4
REF_Y = (0.12, 1.2)   # reference Morse of the y basis, re = 1.8


def _torch():
    import torch

    return torch


def _st(t):
    return _torch().cuda.current_stream(t.device).cuda_stream


def gemm(A, B, C=None, ta=False, tb=False, alpha=1.0, beta=0.0):
    """C = alpha op(A) op(B) + beta C on row-major 2-D CUDA tensors (f32 or f64)."""
    torch = _torch()
    M = A.shape[1] if ta else A.shape[0]
    K = A.shape[0] if ta else A.shape[1]
    Nn = B.shape[0] if tb else B.shape[1]
    assert (B.shape[1] if tb else B.shape[0]) == K
    if C is None:
        C = torch.empty((M, Nn), dtype=A.dtype, device=A.device)
    fn = N.load().espec_gemm_f64 if A.dtype == torch.float64 else N.load().espec_gemm_f32
    rc = fn(M, Nn, K, alpha, A.data_ptr(), A.shape[1], int(ta), B.data_ptr(), B.shape[1],
            int(tb), beta, C.data_ptr(), C.shape[1], _st(A))
    N.check(rc, "espec_gemm")
    return C


def _morse(q, de, a, re):
    return de * (1.0 - np.exp(-a * (q - re))) ** 2


class ProductBasis:
    """nb x nb products of the nb lowest eigenfunctions of the 1D reference
    Morse Hamiltonian of each axis (the same finite-difference operator, solved
    by the library's eigensolver on an n x 1 grid).  B: [nb*nb, n] float64."""

    def __init__(self, grid, nb=16, device=None):
        torch = _torch()
        dev = device or torch.device("cuda", 0)
        self.grid, self.nb = grid, nb
        nx, ny = grid.np
        x = np.linspace(grid.box[0], grid.box[1], nx)
        y = np.linspace(grid.box[2], grid.box[3], ny)
        sets = []
        for pts, (de, a), re, shm in ((x, REF_X, EG.RE1, grid.shm[0]),
                                      (y, REF_Y, EG.RE2, grid.shm[1])):
            g1 = SimpleNamespace(np=[len(pts), 1], n=len(pts), shm=[shm, 0.0])  # 1D grid
            v = torch.from_numpy(_morse(pts, de, a, re)).to(dev).reshape(1, -1)
            st = EG.lcg_start(len(pts), nb, dev).reshape(1, nb, len(pts))
            r = EG.solve(g1, v, st, nstates=nb, m=40, tol=1e-11, maxrest=400)
            sets.append(r["vec"][0].contiguous())
        self.phi, self.chi = sets
        self.B = torch.empty((nb * nb, grid.n), dtype=torch.float64, device=dev)
        N.check(N.load().espec_outer_basis(self.phi.data_ptr(), nb, nx, self.chi.data_ptr(), nb,
                                           ny, self.B.data_ptr(), _st(self.B)),
                "espec_outer_basis")

    def project(self, vec):
        """vec [P, S, n] -> coefficients [P, S, nb*nb]."""
        P, S, n = vec.shape
        return gemm(vec.reshape(P * S, n), self.B, tb=True).reshape(P, S, -1)

    def expand(self, coef):
        """coefficients [P, S, nb*nb] -> vectors [P, S, n]."""
        P, S, k = coef.shape
        return gemm(coef.reshape(P * S, k).contiguous(), self.B).reshape(P, S, -1)


class MLP:
    """Fully connected tanh network, float32, trained with Adam."""

    def __init__(self, sizes, seed=0, device=None):
        torch = _torch()
        dev = device or torch.device("cuda", 0)
        rng = np.random.default_rng(seed)
        self.sizes = list(sizes)
        self.W, self.b = [], []
        for fi, fo in zip(sizes[:-1], sizes[1:]):
            lim = math.sqrt(6.0 / (fi + fo))  # Glorot uniform
            self.W.append(torch.from_numpy(rng.uniform(-lim, lim, (fi, fo)).astype(np.float32))
                          .to(dev))
            self.b.append(torch.zeros(fo, dtype=torch.float32, device=dev))
        self.params = [p for pair in zip(self.W, self.b) for p in pair]
        self.m1 = [torch.zeros_like(p) for p in self.params]
        self.m2 = [torch.zeros_like(p) for p in self.params]
        self.t = 0

    def forward(self, X):
        acts = [X.contiguous()]
        L = len(self.W)
        for i, (W, b) in enumerate(zip(self.W, self.b)):
            Z = gemm(acts[-1], W)
            N.check(N.load().espec_mlp_bias_act(Z.data_ptr(), b.data_ptr(), Z.shape[0],
                                                Z.shape[1], int(i < L - 1), _st(Z)),
                    "espec_mlp_bias_act")
            acts.append(Z)
        return acts

    def backward(self, acts, dY):
        """Gradients [dW0, db0, dW1, db1, ...] for the loss whose output
        gradient is dY."""
        torch = _torch()
        lib = N.load()
        grads = [None] * len(self.params)
        d = dY
        for i in reversed(range(len(self.W))):
            if i < len(self.W) - 1:  # through tanh: acts[i+1] = tanh(z)
                N.check(lib.espec_mlp_tanh_back(d.data_ptr(), acts[i + 1].data_ptr(), d.numel(),
                                                _st(d)), "espec_mlp_tanh_back")
            dW = gemm(acts[i], d, ta=True)
            db = torch.empty(d.shape[1], dtype=torch.float32, device=d.device)
            N.check(lib.espec_mlp_colsum(d.data_ptr(), d.shape[0], d.shape[1], db.data_ptr(),
                                         _st(d)), "espec_mlp_colsum")
            grads[2 * i], grads[2 * i + 1] = dW, db
            if i > 0:
                d = gemm(d, self.W[i], tb=True)
        return grads

    def loss_grad(self, Y, T):
        torch = _torch()
        dY = torch.empty_like(Y)
        rl = torch.empty(Y.shape[0], dtype=torch.float32, device=Y.device)
        N.check(N.load().espec_mlp_mse(Y.data_ptr(), T.data_ptr(), Y.shape[0], Y.shape[1],
                                       dY.data_ptr(), rl.data_ptr(), _st(Y)), "espec_mlp_mse")
        return rl, dY

    def adam_dev(self, grads, hyper, b1=0.9, b2=0.999, eps=1e-8):
        """Adam with (lr, 1-b1^t, 1-b2^t) in the device tensor hyper."""
        lib = N.load()
        for p, g, m1, m2 in zip(self.params, grads, self.m1, self.m2):
            N.check(lib.espec_mlp_adam_dev(p.data_ptr(), g.data_ptr(), m1.data_ptr(),
                                           m2.data_ptr(), p.numel(), hyper.data_ptr(), b1, b2, eps,
                                           _st(p)), "espec_mlp_adam_dev")

    def adam(self, grads, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        lib = N.load()
        for p, g, m1, m2 in zip(self.params, grads, self.m1, self.m2):
            N.check(lib.espec_mlp_adam(p.data_ptr(), g.data_ptr(), m1.data_ptr(), m2.data_ptr(),
                                       p.numel(), lr, b1, b2, eps, self.t, _st(p)),
                    "espec_mlp_adam")


def normalise(q):
    return (2.0 * (np.asarray(q) - PARAM_LO) / (PARAM_HI - PARAM_LO) - 1.0).astype(np.float32)


class WarmStart:
    """Trains on eigenvectors of the plain solver and proposes start vectors."""

    def __init__(self, grid, nstates=4, nb=16, hidden=(128, 128), m=40, tol=1e-9, maxrest=300,
                 seed=0, device=None):
        torch = _torch()
        self.dev = device or torch.device("cuda", 0)
        self.grid, self.nstates, self.m, self.tol, self.maxrest = grid, nstates, m, tol, maxrest
        self.basis = ProductBasis(grid, nb, self.dev)
        self.nout = nstates * nb * nb
        self.net = MLP([5, *hidden, self.nout], seed=seed, device=self.dev)
        self.scale = 1.0
        self.ref = None

    # -- the plain solver --------------------------------------------------
    def potentials(self, q):
        torch = _torch()
        return EG.morse2d_potentials(self.grid, torch.as_tensor(np.asarray(q), dtype=torch.float64,
                                                                device=self.dev))

    def cold_start(self, P):
        st = EG.lcg_start(self.grid.n, self.nstates, self.dev)
        return st.expand(P, self.nstates, self.grid.n).contiguous()

    def solve(self, q, start=None, batch=1024):
        """Eigensolve of every parameter set (cold start when start is None);
        problems are solved in batches of `batch` CTAs."""
        torch = _torch()
        q = np.asarray(q)
        outs = []
        for a in range(0, len(q), batch):
            qq = q[a:a + batch]
            st = self.cold_start(len(qq)) if start is None else start[a:a + batch].contiguous()
            outs.append(EG.solve(self.grid, self.potentials(qq), st, nstates=self.nstates,
                                 m=self.m, tol=self.tol, maxrest=self.maxrest))
        return {k: torch.cat([o[k] for o in outs]) for k in outs[0]}

    # -- training ----------------------------------------------------------
    def targets(self, vec):
        """Coefficients of the solver's eigenvectors with one sign convention
        per state: positive overlap with the first training sample."""
        torch = _torch()
        c = self.basis.project(vec)  # [P, S, nb^2] float64
        if self.ref is None:
            self.ref = c[0].clone()
        ov = (c * self.ref.unsqueeze(0)).sum(-1)  # sign bookkeeping of the data set
        c = c * torch.where(ov < 0, -1.0, 1.0).unsqueeze(-1)
        return c

    def fit(self, q, vec, epochs=400, batch=256, lr=2e-3, lr_min=2e-5, seed=1, log=None):
        torch = _torch()
        c = self.targets(vec).reshape(len(q), -1)
        rms = float(torch.sqrt((c * c).mean()).item())
        self.scale = 1.0 / rms
        T = torch.empty(c.shape, dtype=torch.float32, device=self.dev)
        N.check(N.load().espec_convert(c.data_ptr(), T.data_ptr(), c.numel(), 1, self.scale,
                                       _st(c)), "espec_convert")
        X = torch.from_numpy(normalise(q)).to(self.dev)
        rng = np.random.default_rng(seed)
        P = len(q)
        batch = min(batch, P)
        nsteps = epochs * max(1, P // batch)
        b1, b2 = 0.9, 0.999
        # one training step (gather, forward, loss, backward, Adam) captured in
        # a CUDA graph; per replay only the batch indices and the Adam
        # hyper-parameters change, both written into device buffers
        idx = torch.zeros(batch, dtype=torch.long, device=self.dev)
        hyper = torch.tensor([lr, 1.0 - b1, 1.0 - b2], dtype=torch.float32, device=self.dev)
        xb = torch.empty((batch, X.shape[1]), dtype=torch.float32, device=self.dev)
        tb = torch.empty((batch, T.shape[1]), dtype=torch.float32, device=self.dev)

        def body():
            torch.index_select(X, 0, idx, out=xb)
            torch.index_select(T, 0, idx, out=tb)
            acts = self.net.forward(xb)
            rl, dY = self.net.loss_grad(acts[-1], tb)
            self.net.adam_dev(self.net.backward(acts, dY), hyper, b1, b2)
            return rl

        # warm-up on a side stream (required before capture); its Adam step is
        # undone by resetting the moments below
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        saved = [p.clone() for p in self.net.params]
        with torch.cuda.stream(s):
            body()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            rl = body()
        for p, p0, m1, m2 in zip(self.net.params, saved, self.net.m1, self.net.m2):
            p.copy_(p0)
            m1.zero_()
            m2.zero_()
        # cosine learning-rate schedule and Adam bias corrections of every step
        t = np.arange(1, nsteps + 1, dtype=np.float64)
        lr_t = lr_min + 0.5 * (lr - lr_min) * (1.0 + np.cos(np.pi * (t - 1) / max(1, nsteps - 1)))
        sched = torch.from_numpy(np.stack([lr_t, 1.0 - b1 ** t, 1.0 - b2 ** t], 1)
                                 .astype(np.float32)).to(self.dev)
        step = 0
        hist = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(P)).to(self.dev)
            for a in range(0, P - batch + 1, batch):
                idx.copy_(perm[a:a + batch])
                hyper.copy_(sched[step])
                graph.replay()
                step += 1
            if log is not None and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                hist.append((ep, float(rl.sum().item())))
                log(ep, hist[-1][1])
        self.net.t = step
        del graph
        return hist

    # -- inference ---------------------------------------------------------
    def propose(self, q):
        """Start vectors [P, nstates, n] (float64) for the parameter sets q."""
        torch = _torch()
        X = torch.from_numpy(normalise(q)).to(self.dev)
        Y = self.net.forward(X)[-1]
        c = torch.empty(Y.shape, dtype=torch.float64, device=self.dev)
        N.check(N.load().espec_convert(Y.data_ptr(), c.data_ptr(), Y.numel(), 0, 1.0 / self.scale,
                                       _st(Y)), "espec_convert")
        return self.basis.expand(c.reshape(len(q), self.nstates, -1))

    def solve_warm(self, q):
        """Warm-started solve; problems that did not reach the tolerance are
        solved again from the cold start and their H*v counts added."""
        torch = _torch()
        r = self.solve(q, start=self.propose(q))
        bad = (r["resid"] > self.tol).any(dim=1).nonzero().flatten().cpu().numpy()
        r["fallback"] = len(bad)
        if len(bad):
            rc = self.solve(np.asarray(q)[bad])
            for k in ("eval", "vec", "resid"):
                r[k][bad] = rc[k]
            r["matvecs"][bad] += rc["matvecs"]
        return r


def sample_params(P, seed):
    rng = np.random.default_rng(seed)
    return PARAM_LO + (PARAM_HI - PARAM_LO) * rng.random((P, 5))
