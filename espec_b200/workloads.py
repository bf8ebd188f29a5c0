"""Synthetic workloads with the shapes of the benchmark configurations.

No dataset is involved: every input is generated from the stated formulas
(seeded where random).  Units: bohr, hartree, electron masses, fs.
"""
import numpy as np

SHFS = 2.4188843243e-2  # fs per atomic time unit
SCAN_SIZES = (256, 384, 512, 768, 1024, 1536, 2048)


def morse(x, de, a, re):
    return de * (1.0 - np.exp(-a * (x - re))) ** 2


def gaussian(x, x0, sigma):
    g = np.exp(-((x - x0) ** 2) / (2.0 * sigma ** 2))
    return g / np.sqrt(np.sum(g * g))  # eSPec normalisation: sum |psi|^2 = 1


def morse1d(n=1024, x0=0.5, x1=8.0, de=0.17, a=1.0, re=1.4, mass=918.0, center=1.8,
            sigma=0.2, dt_au=0.5, nsteps=20000):
    """1D Morse split-operator case: N=1024 on [0.5, 8] bohr, De=0.17 Eh,
    a=1 /bohr, re=1.4 bohr, m=918 m_e, Gaussian at 1.8 bohr (sigma 0.2),
    dt = 0.5 au, 20000 steps."""
    x = x0 + np.arange(n) * ((x1 - x0) / (n - 1))
    return dict(n=n, x=x, vpot=morse(x, de, a, re), psi=gaussian(x, center, sigma),
                sh=(x1 - x0) / (n - 1), sm=mass, dt_fs=dt_au * SHFS, nsteps=nsteps)


def morse_scan(npk=4096, seed=20261203, x0=0.5, x1=8.0, dt_au=0.5, nsteps=8000, sizes=SCAN_SIZES):
    """Batched 1D Morse scan: npk packets, N ~ U{256..2048 incl. 3*2^k},
    De ~ U[0.05, 0.25] Eh, a ~ U[0.6, 1.6] /bohr, re ~ U[1.0, 2.5] bohr,
    m ~ U[900, 30000] m_e, Gaussian at re + U[-0.3, 0.5] bohr with
    sigma ~ U[0.1, 0.3] bohr, all on [0.5, 8] bohr; dt = 0.5 au."""
    rng = np.random.default_rng(seed)
    n = rng.choice(np.asarray(sizes), size=npk)
    de = rng.uniform(0.05, 0.25, npk)
    a = rng.uniform(0.6, 1.6, npk)
    re = rng.uniform(1.0, 2.5, npk)
    m = rng.uniform(900.0, 30000.0, npk)
    c = re + rng.uniform(-0.3, 0.5, npk)
    s = rng.uniform(0.1, 0.3, npk)
    sh = (x1 - x0) / (n - 1)
    off = np.concatenate([[0], np.cumsum(n)])
    vpot = np.empty(off[-1])
    psi = np.empty(off[-1])
    for k in range(npk):
        x = x0 + np.arange(n[k]) * sh[k]
        vpot[off[k]:off[k + 1]] = morse(x, de[k], a[k], re[k])
        psi[off[k]:off[k + 1]] = gaussian(x, c[k], s[k])
    params = dict(n=n, de=de, a=a, re=re, mass=m, center=c, sigma=s)
    return dict(npk=npk, n=n.astype(np.int32), off=off, sh=sh, sm=m, vpot=vpot, psi=psi,
                dt_fs=dt_au * SHFS, nsteps=nsteps, params=params)
