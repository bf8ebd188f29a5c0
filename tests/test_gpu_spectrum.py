"""GPU parity of the spectrum stage (espec.f:1545-1576, hwhm.f, spectrumtd.f,
cfft.f) against the oracle (FP64, <= 1e-10), against the reference's test 8
golden (print precision) and the executable's printed spectrum text."""
import os

import numpy as np
import pytest
import torch

import espec_b200 as E
from espec_b200 import spectrum as S
from espec_b200 import workloads as W

import golden_cases as G

pytestmark = pytest.mark.gpu


def load_test8():
    d = G.load("test8")
    m = G.manifest()["test8"]
    cin = d["cin"]
    dtf = cin[1, 0] - cin[0, 0]
    tf = cin[-1, 0] + dtf
    return d, m, cin, dtf, tf


def test_test8_dropins_match_oracle_golden_and_text(oracle, capfd):
    d, m, cin, dtf, tf = load_test8()
    mf = m["mf"]
    chwhm, de, e1i, ade = m["hwhm"]
    u = np.ascontiguousarray(cin[:, 1])
    v = np.ascontiguousarray(cin[:, 2])
    ru, rv = oracle.hwhm(mf, dtf, tf, chwhm, de - e1i, u, v)
    en, su, sv = oracle.spectrumtd(False, mf, dtf, tf, 1e-3, ade, ru, rv, quirks=16)
    tal = S.hwhm(mf, dtf, tf, chwhm, de - e1i, u, v)
    assert tal == chwhm * 1.5192676
    assert np.max(np.abs(u - ru)) <= 1e-12 and np.max(np.abs(v - rv)) <= 1e-12
    capfd.readouterr()
    de_out = S.spectrumtd(".NONE", mf, dtf, tf, 1e-3, ade, u, v)
    out, _ = capfd.readouterr()
    assert de_out == max(ade, 0.0)
    assert np.max(np.abs(u - su)) <= 1e-10 and np.max(np.abs(v - sv)) <= 1e-10
    n = 1 << mf
    order = np.r_[n // 2:n, 0:n // 2]
    gold = d["spec_golden"]
    assert np.max(np.abs(u[order] - gold[:, 1])) <= 5.1e-8
    assert np.max(np.abs(v[order] - gold[:, 3])) <= 5.1e-8
    lines = out.split("\n")[:-1]
    with open(os.path.join(G.GOLDEN, "test8_spectrum.txt")) as f:
        want = f.read().split("\n")[:-1]
    assert lines[:4] == want[:4]
    rows = lines[4:]
    assert len(rows) == n
    have = rows[:100] + rows[-20:]
    same = 0
    for h, w in zip(have, want[4:]):
        hv, wv = np.array(h.split(), float), np.array(w.split(), float)
        assert np.all(np.abs(hv - wv) <= 1.01e-7), (h, w)
        same += h == w
    assert same >= 110


def test_batched_device_spectra_match_oracle(oracle):
    """C(t) of a batch left on the device -> assembled spectra of every packet."""
    w = W.morse_scan(npk=6, nsteps=2048, seed=11, sizes=(256, 512, 1024))
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="fp64")
    b.load(w["vpot"], w["psi"])
    b.run(w["nsteps"])
    c_host, _ = b.results()
    dev = torch.device("cuda", 0)
    c_dev = torch.from_numpy(c_host).to(dev)
    mf = 12
    dtf = w["dt_fs"]
    tf = (1 << (mf - 1)) * dtf
    for tal, window in [(None, "SG"), (0.05, "SG"), (0.02, None)]:
        for sp in (False, True):
            out = S.spectra(c_dev, mf, dtf, tf, tal=tal, de=0.3, window=window, wp=1e-3,
                            fftnt_sp=sp).cpu().numpy()
            for k in range(6):
                u, v = oracle.total_correlation(mf, c_host[k, : 1 << (mf - 1)])
                if tal is not None:
                    u, v = oracle.hwhm(mf, dtf, tf, tal, 0.3, u, v)
                _, su, sv = oracle.spectrumtd(window == "SG", mf, dtf, tf, 1e-3, 0.0, u, v,
                                              quirks=16 if sp else 0)
                ref = su + 1j * sv
                assert np.max(np.abs(out[k] - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
    b.close()


def test_signal_mode_and_sizes(oracle):
    rng = np.random.default_rng(2)
    dev = torch.device("cuda", 0)
    for mf in (0, 1, 2, 5, 10, 14):
        n = 1 << mf
        x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
        out = S.spectra(torch.from_numpy(x).to(dev), mf, 0.01, n * 0.005, assemble=False,
                        window=None).cpu().numpy()
        for k in range(3):
            _, su, sv = oracle.spectrumtd(False, mf, 0.01, n * 0.005, 1e-3, 0.0, x[k].real,
                                          x[k].imag)
            assert np.max(np.abs(out[k] - (su + 1j * sv))) <= 1e-12
