"""The network oracle (oracle/mlp_oracle.py) against finite differences:
its analytic gradients are what the GPU kernels are checked against."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    sizes = [5, 7, 6, 4]
    W = [rng.standard_normal((a, b)) * 0.5 for a, b in zip(sizes[:-1], sizes[1:])]
    b = [rng.standard_normal(s) * 0.1 for s in sizes[1:]]
    X = rng.standard_normal((9, 5))
    T = rng.standard_normal((9, 4))

    def loss():
        return M.mse(M.forward(W, b, X)[-1], T)[0]

    acts = M.forward(W, b, X)
    _, dY = M.mse(acts[-1], T)
    gW, gb = M.backward(W, acts, dY)
    h = 1e-6
    for arrs, grads in ((W, gW), (b, gb)):
        for a, g in zip(arrs, grads):
            for idx in [tuple(rng.integers(0, s) for s in a.shape) for _ in range(6)]:
                old = a[idx]
                a[idx] = old + h
                lp = loss()
                a[idx] = old - h
                lm = loss()
                a[idx] = old
                assert abs((lp - lm) / (2 * h) - g[idx]) <= 1e-7 * max(1.0, abs(g[idx]))


def test_oracle_adam_first_step_is_sign_step():
    w = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -0.25, 1e-3])
    w1, m1, m2 = M.adam(w, g, np.zeros(3), np.zeros(3), 1, 0.01)
    assert np.allclose(w1, w - 0.01 * np.sign(g), atol=1e-6)
