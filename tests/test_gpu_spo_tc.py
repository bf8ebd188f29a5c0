"""The tensor-core variant of 256-point packets (16-point DFT GEMMs on
tcgen05, BF16 x 3 split operands, FP32 accumulation in tensor memory) against
the oracle and against the register-FFT mixed variant.

Its arithmetic is FP32-class, like the other mixed variants: the error
against the FP64 oracle is held to the same bound as the register kernels'
mixed form over the same steps (1e-6, or 8x the batch's FP32-state floor)."""

FLOOR_FACTOR = 8.0


def _bound(w):
    floor = fp32_state_floor(w["n"], w["sh"], w["sm"], w["vpot"], w["psi"], w["off"], 0.5,
                             w["nsteps"])
    return max(1e-6, FLOOR_FACTOR * np.max(floor))
import ctypes as C

import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as N
from espec_b200 import workloads as W
from fp32_floor import fp32_state_floor

pytestmark = pytest.mark.gpu


def _run(w, variant=None):
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="mixed")
    if variant is not None:
        b.set_variant(256, variant)
    b.load(w["vpot"], w["psi"])
    b.run(w["nsteps"])
    c, p = b.results()
    b.close()
    return c, p


def test_tensor_core_variant_matches_oracle_and_register_fft(oracle):
    # 19 packets: two full CTAs of 8 and a partial one
    w = W.morse_scan(npk=19, nsteps=400, seed=21, sizes=(256,))
    c_tc, p_tc = _run(w, N.VARIANT_TC)
    st = C.c_int(-1)
    assert N.load().espec_spo_tc_status(C.byref(st)) == 0 and st.value == 0
    c_rf, _ = _run(w, 0)
    c_ref, u, v = oracle.spo_batch(w["off"], w["sh"], w["sm"], w["vpot"], w["psi"],
                                   np.zeros_like(w["psi"]), w["dt_fs"], w["nsteps"], nthreads=8)
    e_tc = np.max(np.abs(c_tc - c_ref))
    e_rf = np.max(np.abs(c_rf - c_ref))
    assert np.all(np.isfinite(c_tc))
    print("tensor-core |dC|", e_tc, "register-FFT |dC|", e_rf)
    assert e_tc <= _bound(w), (e_tc, e_rf)
    assert np.max(np.abs(p_tc - (u + 1j * v))) <= 5e-5


def test_tensor_core_variant_in_a_mixed_size_batch(oracle):
    w = W.morse_scan(npk=30, nsteps=200, seed=22, sizes=(256, 512, 1024))
    c_tc, _ = _run(w, N.VARIANT_TC)
    c_ref, _, _ = oracle.spo_batch(w["off"], w["sh"], w["sm"], w["vpot"], w["psi"],
                                   np.zeros_like(w["psi"]), w["dt_fs"], w["nsteps"], nthreads=8)
    assert np.max(np.abs(c_tc - c_ref)) <= _bound(w)


def test_tensor_core_variant_refused_outside_its_case():
    w = W.morse_scan(npk=4, nsteps=10, seed=23, sizes=(512,))
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="mixed")
    with pytest.raises(E.EspecError):
        b.set_variant(512, N.VARIANT_TC)
    b.close()
    w = W.morse_scan(npk=4, nsteps=10, seed=23, sizes=(256,))
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision="fp64")
    with pytest.raises(E.EspecError):
        b.set_variant(256, N.VARIANT_TC)
    b.close()
