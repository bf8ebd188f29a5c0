"""Learned warm start for the initial-state eigensolver (no counterpart in the
reference, which starts LANCZSG from its LCG vectors, lanczsc.f:56-62).

A multilayer perceptron (5 -> 3 x 256 GELU -> 4 x 1024) maps the five
parameters of a 2D coupled-Morse potential (De1, a1, De2, a2, lambda) to the
four lowest eigenvectors, written as coefficients in a 32 x 32 sine-DVR
product basis chi_a(x) chi_b(y).  It is trained on eigenvectors that the
plain eigensolver (espec_b200.eig) itself produces over random parameters,
with BF16 weights, activations and gradients as tensor-core GEMM operands,
FP32 accumulation, FP32 master weights and Adam (mlp_tc.cu, mlp.cu).  Its
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

# parameter box around the 2D coupled Morse of the 256 x 256 workload (De =
# 0.17 / 0.12 Eh, a = 1.0 / 1.2 bohr^-1, varied by about +-6 % and +-4 %,
# coupling +-0.01 Eh/bohr^2); inside it the four lowest states
# keep their order (no crossings), so each state is a smooth function of q
PARAM_LO = np.array([0.16, 0.95, 0.11, 1.15, -0.01])
PARAM_HI = np.array([0.18, 1.05, 0.13, 1.25, 0.01])


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


def sine_dvr(n, nb, i0=0, i1=None):
    """nb sine-DVR functions on grid points i0..i1 of an n-point axis, zero
    elsewhere: chi_a(x_i) = sum_j T_ja s_j(i), s_j the particle-in-a-box
    functions vanishing one grid step outside [i0, i1] (orthonormal on the
    grid), T_ja = sqrt(2/(nb+1)) sin(pi j a/(nb+1)) the DVR transform
    (orthogonal).  Returns [nb, n] float64."""
    i1 = n - 1 if i1 is None else i1
    m = i1 - i0 + 1
    j = np.arange(1, nb + 1)
    s = np.zeros((nb, n))
    s[:, i0:i1 + 1] = np.sqrt(2.0 / (m + 1)) * np.sin(np.pi * np.outer(j, np.arange(1, m + 1))
                                                      / (m + 1))
    T = np.sqrt(2.0 / (nb + 1)) * np.sin(np.pi * np.outer(j, j) / (nb + 1))
    return T.T @ s


class SineDVRBasis:
    """nb x nb products chi_a(x) chi_b(y) of sine-DVR functions of each axis;
    project / expand through the separable transform kernel."""

    def __init__(self, grid, nb=32, span=None, device=None):
        torch = _torch()
        dev = device or torch.device("cuda", 0)
        self.grid, self.nb = grid, nb
        nx, ny = grid.np
        span = span or ((0, nx - 1), (0, ny - 1))
        self.phi = torch.from_numpy(sine_dvr(nx, nb, *span[0]).astype(np.float32)).to(dev)
        self.chi = torch.from_numpy(sine_dvr(ny, nb, *span[1]).astype(np.float32)).to(dev)

    def _run(self, direction, psi, c, scale):
        nx, ny = self.grid.np
        N.check(N.load().espec_sep_basis(direction, psi.shape[0] * psi.shape[1], nx, ny, self.nb,
                                         self.phi.data_ptr(), self.chi.data_ptr(),
                                         psi.data_ptr(), c.data_ptr(), float(scale), _st(psi)),
                "espec_sep_basis")

    def project(self, vec, scale=1.0):
        """vec [P, S, n] float64 -> coefficients [P, S, nb*nb] float32."""
        torch = _torch()
        vec = vec.contiguous()
        c = torch.empty((vec.shape[0], vec.shape[1], self.nb * self.nb), dtype=torch.float32,
                        device=vec.device)
        self._run(0, vec, c, scale)
        return c

    def expand(self, coef, scale=1.0):
        """coefficients [P, S, nb*nb] float32 -> vectors [P, S, n] float64."""
        torch = _torch()
        coef = coef.contiguous()
        psi = torch.empty((coef.shape[0], coef.shape[1], self.grid.n), dtype=torch.float64,
                          device=coef.device)
        self._run(1, psi, coef, scale)
        return psi


def gemm_bf16(A, B, C=None, ta=False, tb=False, alpha=1.0, beta=0.0):
    """C (float32) = alpha op(A) op(B) + beta C on the tensor cores; A, B
    bfloat16 row-major 2-D CUDA tensors."""
    torch = _torch()
    M = A.shape[1] if ta else A.shape[0]
    K = A.shape[0] if ta else A.shape[1]
    Nn = B.shape[0] if tb else B.shape[1]
    assert (B.shape[1] if tb else B.shape[0]) == K
    if C is None:
        C = torch.empty((M, Nn), dtype=torch.float32, device=A.device)
    N.check(N.load().espec_gemm_bf16(M, Nn, K, alpha, A.data_ptr(), A.shape[1], int(ta),
                                     B.data_ptr(), B.shape[1], int(tb), beta, C.data_ptr(),
                                     C.shape[1], _st(A)), "espec_gemm_bf16")
    return C


def to_bf16(x, out=None):
    torch = _torch()
    out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device) if out is None else out
    N.check(N.load().espec_to_bf16(x.data_ptr(), out.data_ptr(), x.numel(), _st(x)),
            "espec_to_bf16")
    return out


class MLP:
    """Fully connected GELU network.  FP32 master weights; the products take
    BF16 copies of weights, activations and back-propagated gradients and
    accumulate in FP32 on the tensor cores.  Trained with Adam."""

    def __init__(self, sizes, seed=0, device=None):
        torch = _torch()
        dev = device or torch.device("cuda", 0)
        rng = np.random.default_rng(seed)
        self.sizes = list(sizes)
        self.W, self.b, self.Wb = [], [], []
        for fi, fo in zip(sizes[:-1], sizes[1:]):
            lim = math.sqrt(6.0 / (fi + fo))  # Glorot uniform
            w = torch.from_numpy(rng.uniform(-lim, lim, (fi, fo)).astype(np.float32)).to(dev)
            self.W.append(w)
            self.Wb.append(to_bf16(w))
            self.b.append(torch.zeros(fo, dtype=torch.float32, device=dev))
        self.params = [p for pair in zip(self.W, self.b) for p in pair]
        self.copies = [c for w in self.Wb for c in (w, None)]  # BF16 copy of each parameter
        self.m1 = [torch.zeros_like(p) for p in self.params]
        self.m2 = [torch.zeros_like(p) for p in self.params]

    def forward(self, Xb):
        """Xb [rows, sizes[0]] bfloat16 -> (BF16 layer inputs, FP32 pre-activations);
        the network's output is the last pre-activation."""
        torch = _torch()
        lib = N.load()
        hs, zs = [Xb.contiguous()], []
        L = len(self.W)
        for i, (Wb, b) in enumerate(zip(self.Wb, self.b)):
            Z = gemm_bf16(hs[-1], Wb)
            h = torch.empty(Z.shape, dtype=torch.bfloat16, device=Z.device) if i < L - 1 else None
            N.check(lib.espec_mlp_bias_gelu(Z.data_ptr(), b.data_ptr(), Z.shape[0], Z.shape[1],
                                            int(i < L - 1), h.data_ptr() if h is not None else None,
                                            _st(Z)), "espec_mlp_bias_gelu")
            zs.append(Z)
            if h is not None:
                hs.append(h)
        return hs, zs

    def backward(self, hs, zs, dY):
        """Gradients [dW0, db0, dW1, db1, ...] (FP32) for the loss whose output
        gradient is dY (FP32)."""
        torch = _torch()
        lib = N.load()
        grads = [None] * len(self.params)
        d, db16 = dY, to_bf16(dY)
        for i in reversed(range(len(self.W))):
            dW = gemm_bf16(hs[i], db16, ta=True)
            db = torch.empty(d.shape[1], dtype=torch.float32, device=d.device)
            N.check(lib.espec_mlp_colsum(d.data_ptr(), d.shape[0], d.shape[1], db.data_ptr(),
                                         _st(d)), "espec_mlp_colsum")
            grads[2 * i], grads[2 * i + 1] = dW, db
            if i > 0:
                d = gemm_bf16(db16, self.Wb[i], tb=True)
                db16 = torch.empty(d.shape, dtype=torch.bfloat16, device=d.device)
                N.check(lib.espec_mlp_gelu_back(d.data_ptr(), zs[i - 1].data_ptr(), d.numel(),
                                                db16.data_ptr(), _st(d)), "espec_mlp_gelu_back")
        return grads

    def loss_grad(self, Y, T):
        torch = _torch()
        dY = torch.empty_like(Y)
        rl = torch.empty(Y.shape[0], dtype=torch.float32, device=Y.device)
        N.check(N.load().espec_mlp_mse(Y.data_ptr(), T.data_ptr(), Y.shape[0], Y.shape[1],
                                       dY.data_ptr(), rl.data_ptr(), _st(Y)), "espec_mlp_mse")
        return rl, dY

    def adam(self, grads, hyper, b1=0.9, b2=0.999, eps=1e-8):
        """Adam with (lr, 1-b1^t, 1-b2^t) in the device tensor hyper; refreshes
        the BF16 weight copies."""
        lib = N.load()
        for p, g, m1, m2, cp in zip(self.params, grads, self.m1, self.m2, self.copies):
            N.check(lib.espec_mlp_adam_bf16(p.data_ptr(), g.data_ptr(), m1.data_ptr(),
                                            m2.data_ptr(), p.numel(), hyper.data_ptr(), b1, b2,
                                            eps, cp.data_ptr() if cp is not None else None,
                                            _st(p)), "espec_mlp_adam_bf16")


def normalise(q):
    return (2.0 * (np.asarray(q) - PARAM_LO) / (PARAM_HI - PARAM_LO) - 1.0).astype(np.float32)


class WarmStart:
    """Trains on eigenvectors of the plain solver and proposes start vectors."""

    def __init__(self, grid, nstates=4, nb=32, hidden=(256, 256, 256), m=40, tol=1e-9,
                 maxrest=300, seed=0, span="auto", device=None):
        """span: grid-index ranges ((i0, i1), (j0, j1)) of the DVR functions,
        None for the whole grid, or "auto": the smallest box holding all but
        1e-8 of every training eigenvector's marginal densities (set by fit)."""
        torch = _torch()
        self.dev = device or torch.device("cuda", 0)
        self.grid, self.nstates, self.m, self.tol, self.maxrest = grid, nstates, m, tol, maxrest
        self.nb, self.auto_span = nb, span == "auto"
        self.basis = SineDVRBasis(grid, nb, None if self.auto_span else span, self.dev)
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
    def span_of(self, vec, tail=1e-8, pad=2, sample=256):
        """Grid-index box outside which every sampled eigenvector has less than
        `tail` of its norm along each axis."""
        torch = _torch()
        nx, ny = self.grid.np
        v = vec[:sample].reshape(-1, ny, nx) ** 2
        out = []
        for marg, n in ((v.sum(1), nx), (v.sum(2), ny)):
            marg = marg / marg.sum(1, keepdim=True)
            cum = torch.cumsum(marg, 1).cpu().numpy()
            lo = int((cum > tail).argmax(1).min())
            hi = int((cum < 1.0 - tail).sum(1).max())
            out.append((max(0, lo - pad), min(n - 1, hi + pad)))
        return tuple(out)

    def targets(self, vec):
        """Coefficients of the solver's eigenvectors with one sign convention
        per state: positive overlap with the first training sample."""
        torch = _torch()
        c = self.basis.project(vec)  # [P, S, nb^2] float32
        if self.ref is None:
            self.ref = c[0].clone()
        ov = (c * self.ref.unsqueeze(0)).sum(-1)  # sign bookkeeping of the data set
        c = c * torch.where(ov < 0, -1.0, 1.0).unsqueeze(-1)
        return c

    def fit(self, q, vec, epochs=400, batch=256, lr=2e-3, lr_min=2e-5, seed=1, log=None):
        torch = _torch()
        if self.auto_span:
            self.span = self.span_of(vec)
            self.basis = SineDVRBasis(self.grid, self.nb, self.span, self.dev)
            self.ref = None
        c = self.targets(vec).reshape(len(q), -1)
        rms = float(torch.sqrt((c.double() ** 2).mean()).item())
        self.scale = 1.0 / rms
        T = c * self.scale  # unit-rms targets
        X = to_bf16(torch.from_numpy(normalise(q)).to(self.dev))
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
        xb = torch.empty((batch, X.shape[1]), dtype=torch.bfloat16, device=self.dev)
        tb = torch.empty((batch, T.shape[1]), dtype=torch.float32, device=self.dev)

        def body():
            torch.index_select(X, 0, idx, out=xb)
            torch.index_select(T, 0, idx, out=tb)
            hs, zs = self.net.forward(xb)
            rl, dY = self.net.loss_grad(zs[-1], tb)
            self.net.adam(self.net.backward(hs, zs, dY), hyper, b1, b2)
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
        for w, wb in zip(self.net.W, self.net.Wb):
            to_bf16(w, wb)
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
        del graph
        return hist

    # -- inference ---------------------------------------------------------
    def propose(self, q):
        """Start vectors [P, nstates, n] (float64) for the parameter sets q."""
        torch = _torch()
        Xb = to_bf16(torch.from_numpy(normalise(q)).to(self.dev))
        Y = self.net.forward(Xb)[1][-1]
        return self.basis.expand(Y.reshape(len(q), self.nstates, -1), 1.0 / self.scale)

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
