"""Oracle checks of the rotation-axis search (CPU only).

The oracle restates AverageGradient::apply (ctas src/common/lct.cpp:863-913),
the projection-pair error (lct.cpp:1246-1252) and the raxis() control flow
(lct.cpp:1114-1297).  These tests check the restatement against independent
numpy forms of the same definitions: the FFT-product smoothing the reference
computes, the blitz range rules of the derivative statements, and the
full-array-to-view assignment of the gradient magnitude.  (The metric itself
is pinned to the reference's code in tests/test_lct_pin.py.)
"""
import numpy as np
import pytest

import oracle as O
from ctas_b200 import phantom as ph


def _metric_numpy(S, centre, sigma):
    """AverageGradient::apply on a given slice, written with numpy FFTs and
    array slicing (an independent form of the oracle's loops)."""
    W = S.shape[0]
    if sigma > 1:
        sig22 = np.float32(2) * np.float32(sigma) * np.float32(sigma)
        a = np.arange(W)
        g = np.exp((-(a[:, None] ** 2 + a[None, :] ** 2)).astype(np.float32) / sig22).astype(np.float32)
        B = np.real(np.fft.ifft2(np.fft.fft2(S.astype(np.float64)) * np.fft.fft2(g.astype(np.float64))))
        B = B.astype(np.float32)
    else:
        B = S.astype(np.float32)
    # ceil(abs(c)) with the C library's int abs() in ct.h:277: |trunc(c)|
    cc = abs(int(np.float32(centre)))
    R = W - 2 * cc
    Cv = B[cc:cc + R]
    dH = np.zeros((W, W), np.float32)
    dV = np.zeros((W, W), np.float32)

    def acc(D, s0, s1, k):
        dst = D[cc:cc + R]
        r0, r1 = max(0, s0), R - 1 + min(0, s0)
        c0, c1 = max(0, s1), W - 1 + min(0, s1)
        dst[r0:r1 + 1, c0:c1 + 1] = (dst[r0:r1 + 1, c0:c1 + 1]
                                     + np.float32(k) * Cv[r0 - s0:r1 - s0 + 1, c0 - s1:c1 - s1 + 1])

    for s0, s1, k in [(-1, -1, -1), (-1, 0, -2), (-1, 1, -1), (1, -1, 1), (1, 0, 2), (1, 1, 1)]:
        acc(dH, s0, s1, k)
    for s0, s1, k in [(-1, -1, -1), (0, -1, -2), (1, -1, -1), (-1, 1, 1), (0, 1, 2), (1, 1, 1)]:
        acc(dV, s0, s1, k)
    # the R x W view receives the first R rows of the full-size arrays
    M = np.sqrt(dH[:R] * dH[:R] + dV[:R] * dV[:R]).astype(np.float32)
    M[:, 0] = 0
    M[:, W - 1] = 0
    M[0, :] = 0
    M[R - 1, :] = 0
    s = float(np.sum(M.astype(np.float64)))
    n = int(np.count_nonzero(M > 0))
    if sigma > 1:  # the reference's FFT noise makes every region magnitude positive
        region = np.zeros((R, W), bool)
        region[max(cc, 1):R - 1, 1:W - 1] = True
        n = int(np.count_nonzero(region | (M > 0)))
    return np.float32(np.float32(s) / np.float32(n)) if n else np.float32(0), s, n


@pytest.mark.parametrize("W,centre,sigma", [(48, 0.0, 0.5), (48, 2.3, 0.5), (64, -3.5, 1.7),
                                            (64, 5.0, 2.5), (40, 1.0, 1.2)])
def test_ag_metric_matches_numpy_form(W, centre, sigma):
    rng = np.random.default_rng(W + int(10 * sigma))
    S = rng.standard_normal((W, W)).astype(np.float32)
    S[:, :2] = 0  # some exact zeros, as outside the reconstruction disc
    v, s, n = O.ag_metric(S, centre, sigma)
    vn, sn, nn = _metric_numpy(S, centre, sigma)
    assert n == nn
    assert abs(s - sn) <= 1e-5 * abs(sn)
    assert abs(float(v) - float(vn)) <= 1e-5 * abs(float(vn))


def test_ag_metric_row_offset_quirk():
    """The magnitude rows are offset by the crop: a slice whose only structure
    is in the bottom rows of the crop contributes nothing, because the cropped
    view takes the first R rows of the full-size derivative arrays."""
    W, centre = 40, 4.0  # crop 4 rows top and bottom, R = 32
    S = np.zeros((W, W), np.float32)
    S[33:36, 10:30] = 1.0  # rows 29..31 of the crop: derivatives land in full rows 32..36
    v, s, n = O.ag_metric(S, centre, 0.5)
    assert n == 0 and s == 0.0 and v == 0.0
    S2 = np.zeros((W, W), np.float32)
    S2[12:14, 10:30] = 1.0
    assert O.ag_metric(S2, centre, 0.5)[2] > 0


@pytest.mark.parametrize("xs", [-7, -1, 0, 3, 20])
def test_pair_sq_matches_numpy(xs):
    rng = np.random.default_rng(xs + 50)
    rows, W = 3, 37
    p0 = rng.random((rows, W), dtype=np.float32)
    p1 = rng.random((rows, W), dtype=np.float32)
    aver = np.float32(0.375)
    dlt = np.full((rows, W), aver, np.float32)
    R = p1[:, ::-1]
    d0, d1 = max(0, xs), W - 1 + min(0, xs)
    s0 = max(0, -xs)
    dlt[:, d0:d1 + 1] = R[:, s0:s0 + (d1 - d0 + 1)]
    dlt = (dlt - p0).astype(np.float32)
    want = float(np.sum((dlt * dlt).astype(np.float32).astype(np.float64)))
    got = O.lib().orc_pair_sq(p0, p1, rows, W, aver, xs)
    assert abs(got - want) <= 1e-12 * want


def test_raxis_pair_finds_mirror_axis():
    """Two opposite projections of a profile mirrored about axis a: the pair
    method returns a to within its bisection tolerance (0.5 px)."""
    W, rows = 256, 2
    x = np.arange(W, dtype=np.float64)
    for a in (127.5, 131.0, 120.25):
        f = lambda t: 1.0 + 0.5 * np.exp(-((t - 90) / 12) ** 2) + 0.3 * np.exp(-((t - 170) / 20) ** 2)
        p0 = np.tile(f(x), (rows, 1)).astype(np.float32)
        p180 = np.tile(f(2 * a - x), (rows, 1)).astype(np.float32)
        got = O.raxis_pair(p0, p180, 0.1)
        assert abs(float(got) - a) <= 0.5 + 1e-3, (a, got)


def test_raxis_search_restatement_finds_axis():
    """The full search (algorithm 1) on an exact phantom with a shifted axis
    lands within a pixel of the true axis."""
    W, N, c_true = 96, 61, 2.0
    el = ph.random_ellipses(7, 6, W, axes=(4, 20))
    p = ph.sinogram(el, N, W, center=c_true)
    T = np.exp(-p * (0.5 / max(1e-6, float(p.max())))).astype(np.float32)
    axis, calls = O.raxis(T, 180.0, 0.25, 1)
    assert calls >= 3
    assert abs(float(axis) - (0.5 * (W - 1) + c_true)) <= 1.5, axis
