"""GPU test of espec_spo_run_static, the entry point that allocates nothing.

It is meant for callers that cannot call cudaMalloc (an application that
owns the whole device memory pool, a fixed memory budget, or code running
while other work is being captured).  The test calls it through the C-ABI
twice in a row, with different packets each time (the second call must not
see anything of the first in the shared scratch array), and compares C(t)
and psi(TF) with the plan-based entry point (same kernel variant) within
the tolerances of the other GPU tests.  This file is collected last so a run
that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan_reference(E, w, precision):
    b = E.SpoBatch(w["n"], w["sh"], w["sm"], w["dt_fs"], precision=precision)
    for size in set(int(x) for x in w["n"]):
        b.set_variant(size, 0)
    b.load(w["vpot"], w["psi"])
    b.run(w["nsteps"])
    c, p = b.results()
    b.close()
    return c, p


def _static_buffers(w, torch):
    """Device inputs and outputs of one call, allocated by the test (the
    entry point itself allocates nothing)."""
    dev = torch.device("cuda")
    npk = int(w["npk"])
    ns = int(w["nsteps"])
    v = torch.from_numpy(np.ascontiguousarray(w["vpot"])).to(dev)
    psi = np.zeros(2 * w["psi"].size)
    psi[0::2] = w["psi"]
    p0 = torch.from_numpy(psi).to(dev)
    c_out = torch.full((2 * npk * (ns + 1),), np.nan, dtype=torch.float64, device=dev)
    p_out = torch.full((2 * w["psi"].size,), np.nan, dtype=torch.float64, device=dev)
    return v, p0, c_out, p_out


def _static_run(lib, w, precision, torch, bufs):
    v, p0, c_out, p_out = bufs
    npk = int(w["npk"])
    ns = int(w["nsteps"])
    n = np.ascontiguousarray(w["n"], dtype=np.int32)
    sh = np.ascontiguousarray(w["sh"], dtype=np.float64)
    sm = np.ascontiguousarray(w["sm"], dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.espec_spo_run_static(npk, n.ctypes.data_as(C.POINTER(C.c_int)),
                                  sh.ctypes.data_as(C.POINTER(C.c_double)),
                                  sm.ctypes.data_as(C.POINTER(C.c_double)), w["dt_fs"],
                                  precision, v.data_ptr(), p0.data_ptr(), ns, c_out.data_ptr(),
                                  p_out.data_ptr(), stream)
    assert rc == 0, lib.espec_last_error()
    torch.cuda.synchronize()


def _static_read(w, bufs):
    npk = int(w["npk"])
    ns = int(w["nsteps"])
    c = bufs[2].cpu().numpy()
    p = bufs[3].cpu().numpy()
    return (c[0::2] + 1j * c[1::2]).reshape(npk, ns + 1), p[0::2] + 1j * p[1::2]


def _static_call(lib, w, precision, torch):
    bufs = _static_buffers(w, torch)
    _static_run(lib, w, precision, torch, bufs)
    return _static_read(w, bufs)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 5e-6)])
def test_static_entry_matches_plan_entry_on_two_calls(precision, tol):
    torch = pytest.importorskip("torch")
    import espec_b200 as E
    from espec_b200 import _native as N
    from espec_b200 import workloads as W

    lib = N.load()
    prec = {"fp64": N.FP64, "mixed": N.MIXED}[precision]
    calls = [W.morse_scan(npk=12, nsteps=300, seed=41, sizes=(1024, 384, 2048, 256)),
             W.morse_scan(npk=9, nsteps=250, seed=42, sizes=(768, 512, 1536, 4096))]
    for w in calls:
        assert int(w["off"][-1]) <= 32768
        c, p = _static_call(lib, w, prec, torch)
        c_ref, p_ref = _plan_reference(E, w, precision)
        assert np.all(np.isfinite(c)) and np.all(np.isfinite(p))
        assert np.max(np.abs(c - c_ref)) <= tol
        assert np.max(np.abs(p - p_ref)) <= tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 5e-6)])
def test_static_entry_at_its_limit_allocates_nothing(precision, tol):
    """128 packets of 256 points (exactly the 32768-point, 128-packet limit of
    the scratch layout).  The first call may load kernels; the free device
    memory seen by cudaMemGetInfo around the second, identical call must not
    move."""
    torch = pytest.importorskip("torch")
    import espec_b200 as E
    from espec_b200 import _native as N
    from espec_b200 import workloads as W

    lib = N.load()
    prec = {"fp64": N.FP64, "mixed": N.MIXED}[precision]
    w = W.morse_scan(npk=128, nsteps=120, seed=43, sizes=(256,))
    assert int(w["off"][-1]) == 32768
    bufs = _static_buffers(w, torch)
    _static_run(lib, w, prec, torch, bufs)
    c1, p1 = _static_read(w, bufs)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _static_run(lib, w, prec, torch, bufs)
    free1, _ = torch.cuda.mem_get_info()
    c2, p2 = _static_read(w, bufs)
    c_ref, p_ref = _plan_reference(E, w, precision)
    assert np.array_equal(c1, c2) and np.array_equal(p1, p2)
    assert np.max(np.abs(c2 - c_ref)) <= tol
    assert np.max(np.abs(p2 - p_ref)) <= tol
    assert free1 == free0


def test_static_entry_rejects_sizes_beyond_its_limit():
    from espec_b200 import _native as N

    lib = N.load()
    n = np.full(129, 256, dtype=np.int32)
    sh = np.full(129, 0.01)
    rc = lib.espec_spo_run_static(129, n.ctypes.data_as(C.POINTER(C.c_int)),
                                  sh.ctypes.data_as(C.POINTER(C.c_double)),
                                  sh.ctypes.data_as(C.POINTER(C.c_double)), 0.01, N.FP64,
                                  1, 1, 10, 1, None, None)
    assert rc == N.EINVAL
    assert b"128 packets" in lib.espec_last_error()
    n = np.full(9, 4096, dtype=np.int32)
    rc = lib.espec_spo_run_static(9, n.ctypes.data_as(C.POINTER(C.c_int)),
                                  sh.ctypes.data_as(C.POINTER(C.c_double)),
                                  sh.ctypes.data_as(C.POINTER(C.c_double)), 0.01, N.FP64,
                                  1, 1, 10, 1, None, None)
    assert rc == N.EINVAL
    assert b"32768" in lib.espec_last_error()
