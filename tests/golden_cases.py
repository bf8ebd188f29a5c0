"""Load the golden fixtures and turn each into propagation inputs.

The unit conventions follow the reference driver (espec.f): masses in amu are
scaled by 1836.152667539 (espec.f:614), the grid of a .FILE input runs from
its first to its last coordinate with SH = (XF - XI)/(NP - 1) (espec.f:818),
SHM = 1/(24 m SH^2) (espec.f:819), and TF is rounded so that the C(t) stride
LC = 2(TF-TI)/DT / 2^MF is an integer when *CHANGE is on (espec.f:1328-1353).
"""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
AMU = 1836.152667539


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def morse1d_inputs():
    """1D Morse fixture grid, potential and Gaussian (same as make_golden.py)."""
    n = 1024
    x = 0.5 + np.arange(n) * (7.5 / 1023)
    v = 0.17 * (1 - np.exp(-1.0 * (x - 1.4))) ** 2
    psi = np.exp(-((x - 1.8) ** 2) / (2 * 0.2 ** 2))
    psi = psi / np.sqrt(np.sum(psi ** 2))
    rt = lambda a: np.array([float(repr(float(t))) for t in a])
    return rt(x), rt(psi), rt(v)


def lc_and_tf(ti, tf, dt, mf, change=True):
    """espec.f:1328-1353: C(t) stride NC and the adjusted final time."""
    while True:
        sc = 2.0 * (tf - ti) / dt
        nc = int(sc / 2.0 ** mf)
        if abs(sc - nc * 2.0 ** mf) >= 1e-10 and change:
            tf = nc * 2.0 ** (mf - 1) * dt
            continue
        return nc, tf


def grid_from_file(coords):
    """(xi, xf, sh) of one axis of a .FILE grid."""
    xi, xf = float(coords[0]), float(coords[-1])
    return xi, xf, (xf - xi) / (len(coords) - 1)


def shm_of(sm, sh):
    # espec.f:819  SHF/(2.4D+1*SM*SMF*SH*SH) with SHF = SMF = 1, left to right
    return 1.0 / ((((24.0 * sm) * 1.0) * sh) * sh)


# reference-defect switches that reproduce the shipped executable per case
QUIRKS_OF = {".PFSPO": 1, ".PSIL": 2, ".PFSOD": 8, ".PSOD": 32}   # oracle.Q_* bits
DIGT_ND = 4


def setup_case(name):
    """Propagation inputs of a golden case, in the reference's conventions."""
    from oracle import oracle as O

    m = manifest()[name]
    d = load(name)
    if m["kind"] == "morse1d":
        x, psi, v = morse1d_inputs()
        np_ = [1024]
        xi, xf, sh = grid_from_file(x)
        shs, xis, xfs = [sh], [xi], [xf]
        sms = [m["mass_amu"] * AMU]
        psi, v = psi, v
    elif m["kind"] == "morse2d":
        np_ = [32, 32]
        gx, gy = grid_from_file(d["x"]), grid_from_file(d["y"])
        xis, xfs, shs = [gx[0], gy[0]], [gx[1], gy[1]], [gx[2], gy[2]]
        sms = [m["mass_amu"][0] * AMU, m["mass_amu"][1] * AMU]
        psi, v = d["psi"].reshape(-1), d["v"].reshape(-1)
    elif m["kind"] == "test4":
        np_ = [201]
        xi, xf, sh = grid_from_file(d["x"])
        shs, xis, xfs = [sh], [xi], [xf]
        sms = [m["mass_amu"] * AMU]
        psi = d["psi"]
        v = d["v"] - d["v"].min()  # *SHIFT_POTENTIAL default on (rdpt.f)
    else:
        raise KeyError(name)
    ti = m.get("ti_fs", 0.0)
    lc, tf = lc_and_tf(ti, m["tf_fs"], m["dt_fs"], m["mf"])
    absorb, vabc = O.ABS_NONE, None
    if m.get("absorb") == "VOPTIC_POLIN":
        absorb = O.ABS_VOPTIC
        vabc = O.absorbingbc(np_, O.ABC_VOPTIC_POLIN, [m["al"]], [m["ar"]], shs, xis, xfs,
                             m["voi"] + [0.0])
    elif m.get("absorb") == "SMOOTHW":
        absorb = O.ABS_SMOOTHW
        vabc = O.absorbingbc(np_, O.ABC_SMOOTHW, [m["al"]], [m["ar"]], shs, xis, xfs,
                             m["voi"] + [0.0])
    quirks = QUIRKS_OF[m["prop"]] | (DIGT_ND if len(np_) > 1 else 0)
    return dict(meta=m, data=d, np=np_, sh=shs, sm=sms, shm=[shm_of(a, b) for a, b in zip(sms, shs)],
                xi=xis, xf=xfs, dt=m["dt_fs"], ti=ti, tf=tf, lc=lc, vpot=v, psi=psi, vabc=vabc,
                absorb=absorb, ref_quirks=quirks, tol=m.get("tol", 1e3), mp=m.get("mp", 10))


def run_oracle(case, quirks, prtcrl=1):
    from oracle import oracle as O

    p = O.make_prop(case["np"], case["dt"], case["ti"], case["tf"], case["sh"], case["sm"],
                    lc=case["lc"], tol=case["tol"], absorb=case["absorb"], prtcrl=prtcrl,
                    quirks=quirks, mp=case["mp"], change=1, shm=case["shm"])
    fn = {".PFSPO": O.pspofft, ".PFSOD": O.psodfft, ".PSIL": O.plnz,
          ".PSOD": O.psod}[case["meta"]["prop"]]
    return fn(p, case["vpot"], case["psi"], np.zeros_like(case["psi"]), vabc=case["vabc"])
