"""The network oracle (oracle/mlp_oracle.py) against finite differences and
textbook identities: its analytic gradients, Adam step, bfloat16 rounding and
sine-DVR basis are what the GPU kernels are checked against."""
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
        return M.mse(M.forward(W, b, X)[1][-1], T)[0]

    hs, zs = M.forward(W, b, X)
    _, dY = M.mse(zs[-1], T)
    gW, gb = M.backward(W, hs, zs, dY)
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


def test_gelu_derivative():
    z = np.linspace(-6, 6, 101)
    h = 1e-6
    fd = (M.gelu(z + h) - M.gelu(z - h)) / (2 * h)
    assert np.max(np.abs(fd - M.gelu_grad(z))) <= 1e-8
    assert abs(M.gelu(1.0) - 0.8413447460685429) <= 1e-15  # 1 * Phi(1)


def test_oracle_adam_first_step_is_sign_step():
    w = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -0.25, 1e-3])
    w1, m1, m2 = M.adam(w, g, np.zeros(3), np.zeros(3), 1, 0.01)
    assert np.allclose(w1, w - 0.01 * np.sign(g), atol=1e-6)


def test_bf16_rounding():
    # 1 + 2^-8 is halfway between bfloat16 neighbours 1 and 1 + 2^-7: ties to even
    assert M.bf16(1.0 + 2.0 ** -8) == 1.0
    assert M.bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6
    assert M.bf16(-3.0) == -3.0
    x = np.random.default_rng(1).standard_normal(1000)
    assert np.max(np.abs(M.bf16(x) - x) / np.abs(x)) <= 2.0 ** -8  # half a unit in the 8th bit


def test_sine_dvr_is_orthonormal_and_separable_transform_inverts():
    phi = M.sine_dvr(40, 12)
    chi = M.sine_dvr(36, 12, 3, 30)
    assert np.allclose(phi @ phi.T, np.eye(12), atol=1e-13)
    assert np.allclose(chi @ chi.T, np.eye(12), atol=1e-13)
    assert np.all(chi[:, :3] == 0) and np.all(chi[:, 31:] == 0)
    c = np.random.default_rng(2).standard_normal(144)
    assert np.allclose(M.project(phi, chi, M.expand(phi, chi, c)), c, atol=1e-12)
