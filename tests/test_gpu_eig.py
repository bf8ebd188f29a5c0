"""GPU parity of the batched initial-state eigensolver (LANCZSG with locking
and the true residual) against the oracle's restatement: eigenvalues to
1e-9 Eh, residuals <= tol, the same eigenvectors, H*v counts within one
restart; and of its LCG start vectors and potentials."""
import numpy as np
import pytest
import torch

from espec_b200 import eig as EG

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def test_lcg_start_matches_oracle(oracle):
    got = EG.lcg_start(1000, 4, DEV).cpu().numpy()
    assert np.array_equal(got, oracle.lcg_start(1000, 4))


def test_potentials_match_numpy():
    g = EG.Grid2D((33, 29))
    q = torch.tensor([[0.17, 1.0, 0.12, 1.2, 0.01], [0.2, 0.9, 0.1, 1.3, -0.015]],
                     dtype=torch.float64, device=DEV)
    v = EG.morse2d_potentials(g, q).cpu().numpy()
    x = np.linspace(g.box[0], g.box[1], 33)
    y = np.linspace(g.box[2], g.box[3], 29)
    X, Y = np.meshgrid(x, y, indexing="ij")
    for k, (d1, a1, d2, a2, lam) in enumerate(q.cpu().numpy()):
        ref = (d1 * (1 - np.exp(-a1 * (X - 1.4))) ** 2 + d2 * (1 - np.exp(-a2 * (Y - 1.8))) ** 2
               + lam * (X - 1.4) * (Y - 1.8)).ravel(order="F")
        assert np.max(np.abs(v[k] - ref)) <= 1e-14


@pytest.mark.parametrize("np_,m", [((20, 16), 30), ((48, 40), 40)])
def test_eigensolver_matches_oracle(oracle, np_, m):
    g = EG.Grid2D(np_)
    q = torch.tensor([[0.17, 1.0, 0.12, 1.2, 0.01], [0.14, 1.1, 0.15, 1.0, -0.012],
                      [0.2, 0.85, 0.09, 1.35, 0.0]], dtype=torch.float64, device=DEV)
    v = EG.morse2d_potentials(g, q)
    st = EG.lcg_start(g.n, 4, DEV).expand(3, 4, g.n).contiguous()
    r = EG.solve(g, v, st, nstates=4, m=m, tol=1e-9, maxrest=400)
    ev = r["eval"].cpu().numpy()
    vec = r["vec"].cpu().numpy()
    mv = r["matvecs"].cpu().numpy()
    assert np.all(r["resid"].cpu().numpy() <= 1e-9)
    for k in range(3):
        ref = oracle.eig_lanczsg(g.np, g.shm, v[k].cpu().numpy(), 4, m, 1e-9, 400,
                                 st[k].cpu().numpy())
        assert ref["rc"] == 0
        assert np.max(np.abs(ev[k] - ref["evals"])) <= 1e-9
        for s in range(4):
            assert abs(abs(vec[k, s] @ ref["evecs"][s]) - 1.0) <= 1e-7
        assert np.all(np.abs(mv[k] - ref["matvecs"]) <= m + 1), (mv[k], ref["matvecs"])
