"""CPU restatement of the warm-start network (espec_b200/warmstart.py,
espec_b200/csrc/mlp.cu) in float64 numpy: forward, mean-squared-error loss,
backward and one Adam step.

TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels' gradients; the
product never imports it.  The network has no counterpart in eSPec (the
reference starts its eigensolver from LCG vectors), so this restates the
textbook algorithms: tanh layers, MSE loss averaged over all outputs, Adam
(Kingma & Ba, 2015) with bias correction.
"""
import numpy as np


def forward(W, b, X):
    acts = [np.asarray(X, dtype=np.float64)]
    for i, (w, bb) in enumerate(zip(W, b)):
        z = acts[-1] @ w + bb
        acts.append(np.tanh(z) if i < len(W) - 1 else z)
    return acts


def mse(Y, T):
    d = Y - T
    loss = np.sum(d * d) / d.size
    return loss, 2.0 * d / d.size


def backward(W, acts, dY):
    gW, gb = [None] * len(W), [None] * len(W)
    d = dY
    for i in reversed(range(len(W))):
        if i < len(W) - 1:
            d = d * (1.0 - acts[i + 1] ** 2)
        gW[i] = acts[i].T @ d
        gb[i] = d.sum(0)
        if i > 0:
            d = d @ W[i].T
    return gW, gb


def adam(w, g, m1, m2, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    w = w - lr * (m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps)
    return w, m1, m2
