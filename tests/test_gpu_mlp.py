"""GPU kernels of the learned warm start against the CPU oracle: the GEMM
(f64 to 1e-12, f32 to FP32 rounding), the network's forward pass, loss,
gradients and Adam step (float32 kernels vs float64 numpy), and the gain of
the trained network on held-out potentials."""
import numpy as np
import pytest
import torch

from espec_b200 import eig as EG
from espec_b200 import warmstart as WS
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-5)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_gemm_matches_numpy(dtype, tol, ta, tb):
    rng = np.random.default_rng(ta * 2 + tb)
    M_, N_, K = 67, 130, 45
    a = rng.standard_normal((K, M_) if ta else (M_, K))
    b = rng.standard_normal((N_, K) if tb else (K, N_))
    c0 = rng.standard_normal((M_, N_))
    ref = 0.7 * ((a.T if ta else a) @ (b.T if tb else b)) + 0.3 * c0
    A, B = torch.from_numpy(a).to(DEV, dtype), torch.from_numpy(b).to(DEV, dtype)
    C = torch.from_numpy(c0).to(DEV, dtype)
    out = WS.gemm(A, B, C, ta=bool(ta), tb=bool(tb), alpha=0.7, beta=0.3).double().cpu().numpy()
    assert np.max(np.abs(out - ref)) <= tol * np.max(np.abs(ref))


def test_network_gradients_and_adam_match_oracle():
    net = WS.MLP([5, 32, 24, 40], seed=3, device=DEV)
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, (50, 5)).astype(np.float32)
    T = rng.standard_normal((50, 40)).astype(np.float32)
    W = [w.double().cpu().numpy() for w in net.W]
    b = [bb.double().cpu().numpy() for bb in net.b]
    acts = net.forward(torch.from_numpy(X).to(DEV))
    rl, dY = net.loss_grad(acts[-1], torch.from_numpy(T).to(DEV))
    grads = net.backward(acts, dY)
    ref_acts = M.forward(W, b, X)
    loss, rdY = M.mse(ref_acts[-1], T)
    gW, gb = M.backward(W, ref_acts, rdY)
    assert abs(rl.sum().item() - loss) <= 1e-5 * loss
    for a, r in zip(acts[1:], ref_acts[1:]):
        assert np.max(np.abs(a.double().cpu().numpy() - r)) <= 1e-5 * max(1.0, np.max(np.abs(r)))
    for i in range(3):
        for g, r in ((grads[2 * i], gW[i]), (grads[2 * i + 1], gb[i])):
            g = g.double().cpu().numpy()
            assert np.max(np.abs(g - r)) <= 1e-4 * np.max(np.abs(r)), i
    # one Adam step, both forms
    p0 = [p.double().cpu().numpy() for p in net.params]
    gn = [g.double().cpu().numpy() for g in grads]
    net.adam(grads, 1e-3)
    for p, w0, g in zip(net.params, p0, gn):
        w1, _, _ = M.adam(w0, g, np.zeros_like(w0), np.zeros_like(w0), 1, 1e-3)
        assert np.max(np.abs(p.double().cpu().numpy() - w1)) <= 1e-6
    hyper = torch.tensor([1e-3, 1 - 0.9 ** 2, 1 - 0.999 ** 2], dtype=torch.float32, device=DEV)
    net2 = WS.MLP([5, 32, 24, 40], seed=3, device=DEV)
    for p, q in zip(net2.params, net.params):
        p.copy_(q)
    for m, q in zip(net2.m1 + net2.m2, net.m1 + net.m2):
        m.copy_(q)
    net.adam(grads, 1e-3)           # step 2 with host scalars
    net2.adam_dev(grads, hyper)     # step 2 with device hyper-parameters
    for p, q in zip(net.params, net2.params):  # bias corrections rounded differently
        assert float((p - q).abs().max()) <= 1e-7


def test_warm_start_halves_lanczos_iterations():
    """Trained on 1024 eigensolves of a 64 x 64 coupled-Morse family, the
    network's start vectors cut the H*v applications to the 4 lowest states
    of 64 held-out potentials by at least 1.6x, at the same residual
    tolerance and to the same eigenvalues (the full-size figure, 128 x 128
    with 4096 training solves, is reported by bench.py)."""
    g = EG.Grid2D((64, 64))
    ws = WS.WarmStart(g, hidden=(128, 128), seed=0)
    qtr, qte = WS.sample_params(1024, 1), WS.sample_params(64, 2)
    rtr = ws.solve(qtr)
    assert float(rtr["resid"].max()) <= 1e-9
    ws.fit(qtr, rtr["vec"], epochs=1500, batch=128, lr=2e-3)
    cold = ws.solve(qte)
    warm = ws.solve_warm(qte)
    assert float(warm["resid"].max()) <= 1e-9 and float(cold["resid"].max()) <= 1e-9
    assert float((warm["eval"] - cold["eval"]).abs().max()) <= 1e-9
    mc = float(cold["matvecs"].sum(1).double().mean())
    mw = float(warm["matvecs"].sum(1).double().mean())
    assert mc / mw >= 1.6, (mc, mw)
