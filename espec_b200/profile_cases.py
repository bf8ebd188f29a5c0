"""Small, self-checking workloads for profiling single kernels of the library
(one launch each of the kernels named, a few MB on the device):

    python -m espec_b200.profile_cases eig       # eig_kernel: 32 potentials, 128x128, 4 states
    python -m espec_b200.profile_cases spond2d   # x_pass / axis_pass: 256x256 FP64, 20 steps
    python -m espec_b200.profile_cases spond3d   # 128^3 mixed, 10 steps
    python -m espec_b200.profile_cases spectrum  # spec_* kernels: 4096 packets' C(t), 2^13 points
    python -m espec_b200.profile_cases sil       # sil_kernel: 256x256, order 12, 20 steps

Each case exits non-zero if its result is not finite."""
import sys

import numpy as np


def eig():
    import torch

    from espec_b200 import eig as EG
    from espec_b200 import warmstart as WS

    dev = torch.device("cuda", 0)
    g = EG.Grid2D((128, 128))
    q = torch.tensor(WS.sample_params(32, 7), dtype=torch.float64, device=dev)
    v = EG.morse2d_potentials(g, q)
    st = EG.lcg_start(g.n, 4, dev).expand(32, 4, g.n).contiguous()
    r = EG.solve(g, v, st, nstates=4, m=40, tol=1e-9, maxrest=300)
    return float(r["resid"].max())


def _spo_grid(np_, prec, nsteps):
    import espec_b200 as E

    axes = [np.linspace(0.6, 3.6, n) for n in np_]
    G = np.meshgrid(*axes, indexing="ij")
    v = sum(0.15 * (1 - np.exp(-(g - 1.6))) ** 2 for g in G)
    psi = np.exp(-sum((g - 1.9) ** 2 / 0.05 for g in G)).astype(complex)
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2))
    s = E.SpoGrid(np_, [a[1] - a[0] for a in axes], [918.0] * len(np_), 0.5 * 2.4188843243e-2,
                  precision=prec)
    s.load(v.ravel(order="F"), psi.ravel(order="F"))
    s.run(nsteps)
    c, _ = s.results()
    return float(np.abs(c[-1]))


def spectrum():
    import torch

    from espec_b200 import spectrum as S

    dev = torch.device("cuda", 0)
    t = np.arange(4096)[:, None] * 0.01
    c = np.exp(-1j * t * np.linspace(0.1, 0.5, 4096)[None, :]).T.copy()
    out = S.spectra(torch.from_numpy(c).to(dev), 13, 0.01, 4096 * 0.01, tal=0.01, window="SG")
    return float(out.abs().max())


def sil():
    import espec_b200 as E

    n = 256
    x = np.linspace(0.5, 8.0, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    v = 0.17 * (1 - np.exp(-(X - 1.4))) ** 2 + 0.12 * (1 - np.exp(-1.2 * (Y - 1.8))) ** 2
    psi = np.exp(-((X - 1.6) ** 2 + (Y - 2.0) ** 2) / 0.045).astype(complex)
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2))
    h = x[1] - x[0]
    g = E.SilGrid([n, n], [1 / (24 * 918 * h * h), 1 / (24 * 1500 * h * h)], 2.4188843243e-2, 12)
    g.load(v.ravel(order="F"), psi.ravel(order="F"))
    g.run(20)
    c, _ = g.results()
    return float(np.abs(c[-1]))


CASES = {"eig": eig, "spond2d": lambda: _spo_grid([256, 256], "fp64", 20),
         "spond3d": lambda: _spo_grid([128, 128, 128], "mixed", 10), "spectrum": spectrum,
         "sil": sil}

if __name__ == "__main__":
    name = sys.argv[1] if len(sys.argv) > 1 else "eig"
    val = CASES[name]()
    print(name, val)
    sys.exit(0 if np.isfinite(val) else 1)
