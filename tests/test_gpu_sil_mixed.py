"""The mixed form of the short-iterative-Lanczos grid propagator: Lanczos
vectors, residual and H psi in FP32 (the stencil on the residual computed in
FP32), every dot product, the reorthogonalisation coefficients, the Krylov
exponential and the state in FP64.  Its error against the FP64 oracle is an
FP32 rounding walk (a relative 6e-8 per stored vector and stencil), held here
to MIXED_TOL (relative) over 40 steps on random grids and against the
FP64 GPU run on the 256 x 256 workload's grid (measured: 1e-8 to 7e-8)."""
import numpy as np
import pytest

import espec_b200 as E
from espec_b200 import _native as NAT

import golden_cases as G
from test_gpu_sil import oracle_sil, random_packet

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


def run(np_, shm, dt, mp, v, psi, nsteps, precision, absorb=0, vabc=None, quirks=0):
    g = E.SilGrid(np_, shm, dt, mp, absorb=absorb, quirks=quirks, precision=precision)
    g.load(v, psi, vabc=vabc)
    g.run(nsteps)
    c, out = g.results()
    g.close()
    return c, out


@pytest.mark.parametrize("np_,mp,quirks,mask", [
    ([301], 4, 0, False), ([257], 16, 0, True), ([40, 36], 8, 0, True),
    ([12, 10, 8], 6, 0, True), ([9, 7, 11], 12, 0, False)])
def test_mixed_sil_random_grids(oracle, np_, mp, quirks, mask):
    rng = np.random.default_rng(sum(np_) + mp)
    v, psi, sh = random_packet(rng, np_)
    sm = [1000.0 + 400.0 * a for a in range(len(np_))]
    shm = [G.shm_of(m, h) for m, h in zip(sm, sh)]
    vabc = rng.uniform(0.97, 1.0, size=v.size) if mask else None
    absorb = NAT.ABS_SMOOTHW if mask else NAT.ABS_NONE
    dt = 0.02 * NAT.SHFS
    ref, nst = oracle_sil(oracle, np_, sh, sm, shm, dt, 40, v, psi, mp, absorb=absorb,
                          vabc=vabc, quirks=2 if quirks else 0)
    c, out = run(np_, shm, dt, mp, v, psi, nst, "mixed", absorb=absorb, vabc=vabc, quirks=quirks)
    # relative to the largest |C| and |psi| of the run
    psi_ref = ref["u"] + 1j * ref["v"]
    ec = np.max(np.abs(c - ref["c"])) / max(1.0, np.max(np.abs(ref["c"])))
    ep = np.max(np.abs(out - psi_ref)) / max(1.0, np.max(np.abs(psi_ref)))
    print("mixed SIL", np_, mp, "rel |dC|", ec, "rel |dpsi|", ep, "max |psi|",
          np.max(np.abs(psi_ref)))
    assert ec <= MIXED_TOL and ep <= MIXED_TOL, (ec, ep)


def test_mixed_sil_c2_grid_against_fp64():
    """256 x 256 coupled Morse, order 12, 100 steps of dt = 1 au: mixed vs FP64
    on the GPU (the shared-memory form of both)."""
    n = 256
    x = np.linspace(0.5, 8.0, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    morse = lambda q, de, a, re: de * (1 - np.exp(-a * (q - re))) ** 2  # noqa: E731
    V = morse(X, 0.17, 1.0, 1.4) + morse(Y, 0.12, 1.2, 1.8) + 0.01 * (X - 1.4) * (Y - 1.8)
    psi = np.exp(-((X - 1.6) ** 2) / (2 * 0.15 ** 2) - ((Y - 2.0) ** 2) / (2 * 0.15 ** 2))
    psi = (psi / np.sqrt(np.sum(psi ** 2))).ravel(order="F").astype(complex)
    h = x[1] - x[0]
    shm = [G.shm_of(m, h) for m in (918.0, 1500.0)]
    dt = 1.0 * NAT.SHFS
    c64, p64 = run([n, n], shm, dt, 12, V.ravel(order="F"), psi, 100, "fp64")
    c32, p32 = run([n, n], shm, dt, 12, V.ravel(order="F"), psi, 100, "mixed")
    ec, ep = np.max(np.abs(c32 - c64)), np.max(np.abs(p32 - p64))
    print("mixed SIL 256x256 |dC|", ec, "|dpsi|", ep)
    assert ec <= MIXED_TOL and ep <= MIXED_TOL, (ec, ep)


def test_mixed_sil_plan_rules():
    """The mixed form is a SIL option only, without the reference-defect form
    (which grows the state and with it the FP32 rounding); its FP32 basis is
    not exported."""
    import ctypes as C

    lib = NAT.load()
    h = C.c_void_p()
    npa = np.array([64, 1, 1], dtype=np.int32)
    shm = np.array([1.0, 0.0, 0.0])
    rc = lib.espec_grid_create(C.byref(h), NAT.PSOD, 1, npa.ctypes.data_as(C.POINTER(C.c_int)),
                               shm.ctypes.data_as(C.POINTER(C.c_double)), 0.01, 0, NAT.MIXED,
                               0, 0)
    assert rc != 0
    with pytest.raises(E.EspecError):  # the reference-defect form is FP64 only
        E.SilGrid([64], [1.0], 0.01, 4, quirks=NAT.Q_SIL_INPLACE, precision="mixed")
    g = E.SilGrid([64], [1.0], 0.01, 4, precision="mixed")
    x = np.linspace(-1, 1, 64)
    g.load(0.5 * x ** 2, np.exp(-x ** 2 / 0.1).astype(complex))
    g.run(3)
    out = np.zeros(64 * 4)
    assert lib.espec_grid_basis(g._h, 0, out.ctypes.data, 64, NAT.MEM_HOST, None) != 0
    c, _ = g.results()
    assert np.all(np.isfinite(c))
    g.close()
