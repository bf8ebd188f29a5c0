"""CPU checks of bench.py's host-side helpers: spectral peak matching (the
peak-position error reported beside |dC(t)|), the absorbing layer of the
2D/3D legs and the identical workload description of both arms."""
import argparse

import numpy as np

import bench


def _spectra(energies, n, dt, shift=0.0):
    t = np.arange(n) * dt
    c = sum(a * np.exp(-1j * (e + shift) * t) * np.exp(-(t / (0.3 * n * dt)) ** 2)
            for a, e in energies)
    return np.fft.fft(c)[None, :]


def test_peak_error_recovers_a_known_shift():
    n, dt = 4096, 0.5
    lines = [(1.0, 0.1), (0.5, 0.23), (0.3, 0.41)]
    a = _spectra(lines, n, dt)
    b = _spectra(lines, n, dt, shift=2e-5)
    err, count = bench.peak_error_eh(a, b, dt)
    assert count == 3
    assert abs(err - 2e-5) < 2e-6
    same, _ = bench.peak_error_eh(a, a, dt)
    assert same == 0.0


def test_absorbing_layer_is_quadratic_on_the_outer_15_percent():
    q = np.linspace(0.5, 8.0, 256)
    w = bench._box_cap(q)
    assert w[0] == w[-1] == 0.01
    inner = (q > 0.5 + 0.15 * 7.5) & (q < 8.0 - 0.15 * 7.5)
    assert np.all(w[inner] == 0.0)
    assert np.all(np.diff(w[q < 2.0]) <= 0.0)


def test_both_arms_describe_the_same_workload():
    args = argparse.Namespace(npk=4096, nsteps=8000, precision="fp64")
    c = bench.scan_config(args)
    assert c == bench.scan_config(argparse.Namespace(**vars(args)))
    assert c["npk"] == 4096 and c["nsteps"] == 8000 and c["seed"] == bench.SCAN_SEED
