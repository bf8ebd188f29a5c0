"""The grid kernels' point indices: q = (int)(((double)k + 0.5) * (1.0 / nx))
equals k / nx for every grid point k < 2^31 (the kernels' grid_index in
espec_b200/csrc/sil.cu).  The relative rounding error of the two FP64
operations is below 2^-52, so |computed - (k + 0.5)/nx| < (k + 0.5)/nx 2^-52,
far below the 1/(2 nx) distance from (k + 0.5)/nx to the nearest integer.
Checked here in IEEE double arithmetic at every multiple of nx (and its two
neighbours) up to 2^31 for a spread of axis lengths, and exhaustively for
small grids."""
import numpy as np
import pytest


def index_by_multiplication(k, nx):
    inv = np.float64(1.0) / np.float64(nx)
    return ((k.astype(np.float64) + 0.5) * inv).astype(np.int64)


@pytest.mark.parametrize("nx", [1, 2, 3, 7, 9, 10, 12, 32, 33, 36, 40, 48, 64, 96, 100, 127, 128,
                                255, 256, 257, 301, 384, 512, 640, 1000, 1024, 1536, 2047, 2048,
                                4096, 65535, 65536, 700000])
def test_index_exact_at_every_row_boundary(nx):
    q = np.arange(0, (2 ** 31 - 2) // nx, max(1, ((2 ** 31) // nx) // 2000000), dtype=np.int64)
    for off in (-1, 0, 1):
        k = q * nx + off
        k = k[(k >= 0) & (k < 2 ** 31 - 1)]
        np.testing.assert_array_equal(index_by_multiplication(k, nx), k // nx)


@pytest.mark.parametrize("nx,ny", [(32, 32), (10, 12), (100, 96), (48, 33), (256, 256)])
def test_index_exact_on_whole_grids(nx, ny):
    nz = 64
    k = np.arange(nx * ny * nz, dtype=np.int64)
    q = index_by_multiplication(k, nx)
    np.testing.assert_array_equal(q, k // nx)
    z = index_by_multiplication(q, ny)
    np.testing.assert_array_equal(z, k // (nx * ny))
