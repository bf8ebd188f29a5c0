"""CPU restatement of the warm-start network (espec_b200/warmstart.py,
espec_b200/csrc/mlp_tc.cu, espec_b200/csrc/mlp.cu) in float64 numpy: GELU
layers, mean-squared-error loss, backward pass, one Adam step, and the
separable sine-DVR basis transform.

TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels' outputs and
gradients; the product never imports it.  The network has no counterpart in
eSPec (the reference starts its eigensolver from LCG vectors), so this
restates the textbook algorithms: GELU(z) = z Phi(z) (Hendrycks & Gimpel,
2016), MSE loss averaged over all outputs, Adam (Kingma & Ba, 2015) with bias
correction.  With bf16=True every GEMM operand (weights, layer inputs,
back-propagated gradients) is rounded to bfloat16 (round to nearest even) as
the GPU products take them; sums are then exact float64.
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    u = np.asarray(x, dtype=np.float32).copy().view(np.uint32)
    u = (u + np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return u.view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _r(x, on):
    return bf16(x) if on else np.asarray(x, dtype=np.float64)


def forward(W, b, X, bf16_ops=False):
    """Returns (layer inputs h_i, pre-activations z_i); output = z[-1]."""
    hs, zs = [_r(X, bf16_ops)], []
    for i, (w, bb) in enumerate(zip(W, b)):
        z = hs[-1] @ _r(w, bf16_ops) + bb
        zs.append(z)
        if i < len(W) - 1:
            hs.append(_r(gelu(z), bf16_ops))
    return hs, zs


def mse(Y, T):
    d = Y - T
    loss = np.sum(d * d) / d.size
    return loss, 2.0 * d / d.size


def backward(W, hs, zs, dY, bf16_ops=False):
    gW, gb = [None] * len(W), [None] * len(W)
    d = dY
    for i in reversed(range(len(W))):
        dr = _r(d, bf16_ops)
        gW[i] = hs[i].T @ dr
        gb[i] = d.sum(0)
        if i > 0:
            d = (dr @ _r(W[i], bf16_ops).T) * gelu_grad(zs[i - 1])
    return gW, gb


def adam(w, g, m1, m2, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    w = w - lr * (m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps)
    return w, m1, m2


def sine_dvr(n, nb, i0=0, i1=None):
    """nb sine-DVR functions on points i0..i1 of an n-point axis (zero
    elsewhere): the DVR transform sqrt(2/(nb+1)) sin(pi j a/(nb+1)) of the
    particle-in-a-box functions sqrt(2/(m+1)) sin(pi j k/(m+1)), k = 1..m."""
    i1 = n - 1 if i1 is None else i1
    m = i1 - i0 + 1
    out = np.zeros((nb, n))
    for a in range(1, nb + 1):
        for j in range(1, nb + 1):
            t = np.sqrt(2.0 / (nb + 1)) * np.sin(np.pi * j * a / (nb + 1))
            for k in range(1, m + 1):
                out[a - 1, i0 + k - 1] += t * np.sqrt(2.0 / (m + 1)) * np.sin(np.pi * j * k
                                                                                / (m + 1))
    return out


def project(phi, chi, psi):
    """c[a*nb + b] = sum_{x,y} phi[a,x] chi[b,y] psi[x + nx y]."""
    nx, ny = phi.shape[1], chi.shape[1]
    P = np.asarray(psi).reshape(ny, nx)
    return (phi @ P.T @ chi.T).ravel()


def expand(phi, chi, c):
    nb = phi.shape[0]
    C = np.asarray(c).reshape(nb, nb)
    return (phi.T @ C @ chi).T.ravel()
