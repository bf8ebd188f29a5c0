"""The fixed-point slicing of the tensor-core DFT variant (spo_tc.cu), checked
on the host: every slice is exact in BF16, every product order's 32-term sum
is an integer multiple of one power of two that fits FP32 exactly (so the
tensor cores' accumulation cannot round it), and the combined row matches the
exact 16-point DFT to FP32 level."""
import numpy as np

F32 = np.float32
L = 16


def _bf16_exact(x):
    b = np.asarray(x, np.float32).view(np.uint32)
    return bool(np.all((b & 0xFFFF) == 0))


def _slice3(y):
    # spo_tc.cu slice3: round to nearest at 2^-8, 2^-16, 2^-24 in FP32
    a0 = (np.rint(y * F32(256)) * F32(1 / 256)).astype(F32)
    r1 = (y - a0).astype(F32)
    a1 = (np.rint(r1 * F32(65536)) * F32(1 / 65536)).astype(F32)
    r2 = (r1 - a1).astype(F32)
    a2 = (np.rint(r2 * F32(16777216)) * F32(1 / 16777216)).astype(F32)
    return a0, a1, a2


def _dft_real_form():
    # the 32 x 32 real form of the 16-point DFT (build_dft_tiles), both directions
    B = np.zeros((2, 32, 32))
    for d in range(2):
        for nn in range(32):
            for kk in range(32):
                ang = 2 * np.pi * (((nn % L) * (kk % L)) % L) / L
                c, s = np.cos(ang), (-1 if d else 1) * np.sin(ang)
                B[d, nn, kk] = (c if kk < L else -s) if nn < L else (s if kk < L else c)
    return B


def _slice_b(B):
    out, r, sc = [], B.copy(), 256.0
    for _ in range(4):
        bi = np.rint(r * sc) / sc
        r = r - bi
        out.append(bi.astype(F32))
        sc *= 256.0
    return out, r


PRODUCTS = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2), (2, 1), (1, 2), (0, 3)]


def test_dft_slices_are_bf16_and_forward_inverse_to_2e_33():
    B = _dft_real_form()
    bs, r = _slice_b(B)
    assert all(_bf16_exact(b) for b in bs)
    assert np.max(np.abs(r)) <= 2.0 ** -33
    # the sliced forward and inverse matrices are inverses to the residual
    fwd = sum(b[0].astype(np.float64) for b in bs)
    inv = sum(b[1].astype(np.float64) for b in bs)
    assert np.max(np.abs(inv @ fwd / 16 - np.eye(32))) <= 1e-9


def test_every_order_sum_is_exact_in_fp32_and_rows_match_the_dft():
    rng = np.random.default_rng(1)
    B = _dft_real_form()
    bs, _ = _slice_b(B)
    worst = 0.0
    for trial in range(300):
        x = (rng.standard_normal(32) * 10.0 ** rng.uniform(-6, 3)).astype(F32)
        x[rng.random(32) < 0.2] *= F32(1e-5)
        mx = np.abs(x).max()
        e = int(((mx.view(np.int32) >> 23) & 0xFF) - 126)
        y = (x * F32(2.0) ** -e).astype(F32)
        assert 0.5 <= np.abs(y).max() < 1.0
        a = _slice3(y)
        assert all(_bf16_exact(ai) for ai in a)
        d = trial % 2
        P = [np.zeros(32) for _ in range(4)]
        for ia, ib in PRODUCTS:
            o = ia + ib
            terms = a[ia].astype(np.float64)[None, :] * bs[ib][d].astype(np.float64)
            unit = 2.0 ** -(8 * (o + 2))
            assert np.all(terms / unit == np.rint(terms / unit))
            P[o] += terms.sum(axis=1)
        for o in range(4):
            unit = 2.0 ** -(8 * (o + 2))
            assert np.max(np.abs(P[o] / unit)) < 2.0 ** 24
            assert np.all(P[o].astype(F32).astype(np.float64) == P[o])
        p = [q.astype(F32) for q in P]
        out = (p[0] + (p[1] + (p[2] + p[3]))) * F32(2.0) ** e
        exact = B[d] @ x.astype(np.float64)
        worst = max(worst, np.abs(out - exact).max() / (4 * np.linalg.norm(x)))
    # FP32 level relative to the output row's norm (4 |x|)
    assert worst <= 2.0 ** -22, worst
