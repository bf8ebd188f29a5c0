"""GPU kernels of the learned warm start against the CPU oracle: the SIMT
GEMMs (f64 to 1e-12, f32 to FP32 rounding), the tensor-core BF16 GEMM (exact
BF16 inputs, FP32 accumulation), the separable sine-DVR transform, the GELU
network's forward pass, loss, gradients and Adam step against the oracle with
the same BF16 operand rounding, and the gain of the trained network on
held-out potentials."""
import ctypes as C

import numpy as np
import pytest
import torch

from espec_b200 import _native as N
from espec_b200 import eig as EG
from espec_b200 import warmstart as WS
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def tc_status():
    v = C.c_int(-1)
    N.check(N.load().espec_gemm_bf16_status(C.byref(v)), "espec_gemm_bf16_status")
    return v.value


def dev_bf16(a):
    """Upload values that are already bfloat16 numbers (exact conversion)."""
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(DEV).to(torch.bfloat16)


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
    Cc = torch.from_numpy(c0).to(DEV, dtype)
    out = WS.gemm(A, B, Cc, ta=bool(ta), tb=bool(tb), alpha=0.7, beta=0.3).double().cpu().numpy()
    assert np.max(np.abs(out - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("M_,N_,K,ta,tb", [
    (128, 128, 64, 0, 0), (67, 130, 45, 0, 0), (67, 130, 45, 1, 0), (67, 130, 45, 0, 1),
    (67, 130, 45, 1, 1), (300, 256, 1000, 0, 0), (5, 256, 300, 1, 0), (300, 5, 256, 0, 1),
    (256, 4096, 256, 0, 0), (1000, 256, 5, 0, 0), (130, 100, 0, 0, 0), (256, 512, 384, 1, 1),
    (384, 264, 136, 1, 0)])
def test_gemm_bf16_tensor_cores(M_, N_, K, ta, tb):
    rng = np.random.default_rng(M_ + N_ + K + 2 * ta + tb)
    a = M.bf16(rng.standard_normal((K, M_) if ta else (M_, K)))
    b = M.bf16(rng.standard_normal((N_, K) if tb else (K, N_)))
    c0 = rng.standard_normal((M_, N_)).astype(np.float32)
    opa, opb = (a.T if ta else a), (b.T if tb else b)
    ref = 0.7 * (opa @ opb) + 0.3 * c0
    bound = 0.7 * (np.abs(opa) @ np.abs(opb)) * 2.0 ** -22 * max(K, 1) ** 0.5 + 1e-6 * np.abs(ref)
    Cc = torch.from_numpy(c0).to(DEV)
    out = WS.gemm_bf16(dev_bf16(a), dev_bf16(b), Cc, ta=bool(ta), tb=bool(tb), alpha=0.7,
                       beta=0.3).double().cpu().numpy()
    assert tc_status() == 0
    assert np.all(np.abs(out - ref) <= bound + 1e-7), np.max(np.abs(out - ref) - bound)


def test_sep_basis_matches_oracle():
    g = EG.Grid2D((64, 48))
    span = ((2, 60), (0, 47))
    bas = WS.SineDVRBasis(g, 12, span, DEV)
    phi, chi = M.sine_dvr(64, 12, *span[0]), M.sine_dvr(48, 12, *span[1])
    assert np.max(np.abs(bas.phi.double().cpu().numpy() - phi)) <= 1e-7
    rng = np.random.default_rng(5)
    vec = rng.standard_normal((3, 2, g.n))
    c = bas.project(torch.from_numpy(vec).to(DEV), scale=2.0).double().cpu().numpy()
    for p in range(3):
        for s in range(2):
            ref = 2.0 * M.project(phi, chi, vec[p, s])
            assert np.max(np.abs(c[p, s] - ref)) <= 2e-5 * np.max(np.abs(ref))
    coef = rng.standard_normal((3, 2, 144)).astype(np.float32)
    v = bas.expand(torch.from_numpy(coef).to(DEV), scale=0.5).cpu().numpy()
    for p in range(3):
        for s in range(2):
            ref = 0.5 * M.expand(phi, chi, coef[p, s].astype(np.float64))
            assert np.max(np.abs(v[p, s] - ref)) <= 2e-5 * np.max(np.abs(ref))


def test_network_gradients_and_adam_match_oracle():
    sizes = [5, 32, 24, 40]
    net = WS.MLP(sizes, seed=3, device=DEV)
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, (50, 5)).astype(np.float32)
    T = rng.standard_normal((50, 40)).astype(np.float32)
    for bb in net.b:  # non-zero biases
        bb.copy_(torch.from_numpy(rng.standard_normal(bb.shape[0]).astype(np.float32) * 0.1))
    W = [w.double().cpu().numpy() for w in net.W]
    b = [bb.double().cpu().numpy() for bb in net.b]
    hs, zs = net.forward(WS.to_bf16(torch.from_numpy(X).to(DEV)))
    rl, dY = net.loss_grad(zs[-1], torch.from_numpy(T).to(DEV))
    grads = net.backward(hs, zs, dY)
    assert tc_status() == 0
    rh, rz = M.forward(W, b, X, bf16_ops=True)
    loss, rdY = M.mse(rz[-1], T)
    gW, gb = M.backward(W, rh, rz, rdY, bf16_ops=True)
    # FP32 sums against float64 sums can move a BF16 rounding by one unit (2^-8)
    assert abs(rl.sum().item() - loss) <= 1e-3 * loss
    for z, r in zip(zs, rz):
        assert np.max(np.abs(z.double().cpu().numpy() - r)) <= 5e-3 * max(1.0, np.max(np.abs(r)))
    for i in range(3):
        for g, r in ((grads[2 * i], gW[i]), (grads[2 * i + 1], gb[i])):
            g = g.double().cpu().numpy()
            assert np.max(np.abs(g - r)) <= 1e-2 * np.max(np.abs(r)), i
    # one Adam step on the FP32 master weights, BF16 copies refreshed
    p0 = [p.double().cpu().numpy() for p in net.params]
    gn = [g.double().cpu().numpy() for g in grads]
    hyper = torch.tensor([1e-3, 1 - 0.9, 1 - 0.999], dtype=torch.float32, device=DEV)
    net.adam(grads, hyper)
    for p, w0, g in zip(net.params, p0, gn):
        w1, _, _ = M.adam(w0, g, np.zeros_like(w0), np.zeros_like(w0), 1, 1e-3)
        assert np.max(np.abs(p.double().cpu().numpy() - w1)) <= 1e-6
    for w, wb in zip(net.W, net.Wb):
        assert np.array_equal(wb.float().cpu().numpy(), M.bf16(w.cpu().numpy()).astype(np.float32))


def test_warm_start_halves_lanczos_iterations():
    """Trained on 1024 eigensolves of a 64 x 64 coupled-Morse family, the
    network's start vectors (16 x 16 sine-DVR coefficients per state) cut the
    H*v applications to the 4 lowest states of 64 held-out potentials by at
    least 1.6x, at the same residual tolerance and to the same eigenvalues
    (the full-size figure, 128 x 128 with 32 x 32 coefficients, is reported by
    bench.py)."""
    g = EG.Grid2D((64, 64))
    ws = WS.WarmStart(g, nb=16, hidden=(256, 256, 256), seed=0)
    qtr, qte = WS.sample_params(1024, 1), WS.sample_params(64, 2)
    rtr = ws.solve(qtr)
    assert float(rtr["resid"].max()) <= 1e-9
    ws.fit(qtr, rtr["vec"], epochs=1500, batch=128, lr=2e-3)
    cold = ws.solve(qte)
    warm = ws.solve_warm(qte)
    assert tc_status() == 0
    assert float(warm["resid"].max()) <= 1e-9 and float(cold["resid"].max()) <= 1e-9
    assert float((warm["eval"] - cold["eval"]).abs().max()) <= 1e-9
    mc = float(cold["matvecs"].sum(1).double().mean())
    mw = float(warm["matvecs"].sum(1).double().mean())
    assert mc / mw >= 1.6, (mc, mw)
