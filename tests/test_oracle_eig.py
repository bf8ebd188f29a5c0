"""The oracle's initial-state eigensolver (LANCZSG, lanczsc.f:56-120, with
the true residual) against dense diagonalisation of the same finite-
difference Hamiltonian, and its LCG start vectors against rans.f."""
import numpy as np

import golden_cases as G


def morse2d(nx, ny, q, box=(0.6, 3.6, 0.9, 3.9)):
    x = np.linspace(box[0], box[1], nx)
    y = np.linspace(box[2], box[3], ny)
    X, Y = np.meshgrid(x, y, indexing="ij")
    de1, a1, de2, a2, lam = q
    V = (de1 * (1 - np.exp(-a1 * (X - 1.4))) ** 2 + de2 * (1 - np.exp(-a2 * (Y - 1.8))) ** 2
         + lam * (X - 1.4) * (Y - 1.8))
    sh = [x[1] - x[0], y[1] - y[0]]
    shm = [G.shm_of(918.0, sh[0]), G.shm_of(1500.0, sh[1])]
    return V.ravel(order="F"), shm


def dense_h(oracle, np_, shm, v):
    n = int(np.prod(np_))
    H = np.zeros((n, n))
    npa = np.array(list(np_) + [1], dtype=np.int32)
    e = np.zeros(n)
    out = np.zeros(n)
    shma = oracle.f64(list(shm) + [0.0])
    vv = oracle.f64(v)
    for i in range(n):
        e[:] = 0.0
        e[i] = 1.0
        oracle.lib().orc_au(2, oracle._ip(npa), oracle._p(shma), oracle._p(vv), oracle._p(e),
                            oracle._p(out))
        H[:, i] = out
    return H


def test_lcg_start_follows_rans(oracle):
    st = oracle.lcg_start(10, 2)
    seed, seq = 1, []
    for _ in range(30):
        seed = (seed * 1029 + 221591) % 1048576
        seq.append(seed / 1048576)
    assert np.array_equal(st.ravel(), np.array(seq[10:30]))


def test_lanczsg_matches_dense_diagonalisation(oracle):
    np_ = [20, 16]
    v, shm = morse2d(*np_, (0.17, 1.0, 0.12, 1.2, 0.01))
    H = dense_h(oracle, np_, shm, v)
    assert np.allclose(H, H.T, atol=1e-14)
    w, z = np.linalg.eigh(H)
    n = H.shape[0]
    r = oracle.eig_lanczsg(np_, shm, v, 4, 30, 1e-9, 200, oracle.lcg_start(n, 4))
    assert r["rc"] == 0
    assert np.max(np.abs(r["evals"] - w[:4])) <= 1e-9
    assert np.all(r["resid"] <= 1e-9)
    for k in range(4):
        assert abs(abs(r["evecs"][k] @ z[:, k]) - 1.0) <= 1e-8
    assert np.all(r["matvecs"] % 31 == 0)  # whole restarts of m + 1 applications
