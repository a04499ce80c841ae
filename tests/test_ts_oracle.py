"""Oracle checks of the tomosynthesis step ts_add (ctas src/common/lct.cpp:731-787),
CPU only: the oracle's exact row filter against numpy's FFT of the row's own
length (FFTW's R2HC / HC2R pair is the same circular convolution), and the
projection step against a numpy restatement of its float expression."""
import numpy as np
import pytest

import oracle as O


def _ts_numpy(proj, result, ftype, fparam, center, contrast, angle, plane):
    p = proj.astype(np.float32).copy()
    r = result.astype(np.float32).copy()
    rows, n = p.shape
    fw = O.filter_fill_plain(ftype, fparam, n).astype(np.float64)
    if contrast == O.ABS:
        p = (-np.log(p)).astype(np.float32)
    f = np.real(np.fft.ifft(np.fft.fft(p.astype(np.float64), axis=1) * fw[None, :], axis=1))
    p = f.astype(np.float32)
    if contrast == O.REF:
        for x in range(1, n):
            p[:, x] = p[:, x - 1] + p[:, x]
    cs, cc = np.float32(np.sin(np.float32(angle))), np.float32(np.cos(np.float32(angle)))
    plane_cos = np.float32(np.float32(plane) - np.float32(center)) * cs
    rc = np.float32(n * 0.5 + center)
    di = ((np.arange(n, dtype=np.float32) - rc) * cc - plane_cos + rc).astype(np.float32)
    di = np.where(di < 0, np.float32(0), np.where(di >= np.float32(n), np.float32(n - 1), di))
    idx = di.astype(np.int64)
    r = (r + p[:, idx]).astype(np.float32)
    return p, r


@pytest.mark.parametrize("n,contrast,ftype,angle,plane", [
    (64, O.PHS, 1, 0.3, 5), (37, O.ABS, 5, -0.7, -3), (101, O.REF, 6, 1.2, 10),
    (96, O.FLT, 1, 0.0, 0)])
def test_ts_add_matches_numpy_form(n, contrast, ftype, angle, plane):
    rng = np.random.default_rng(n)
    rows = 5
    proj = (rng.random((rows, n)) * 0.8 + 0.1).astype(np.float32)
    res = rng.standard_normal((rows, n)).astype(np.float32)
    p1, r1 = O.ts_add(proj, res, ftype, 0.0, 1.5, contrast, angle, plane)
    p2, r2 = _ts_numpy(proj, res, ftype, 0.0, 1.5, contrast, angle, plane)
    np.testing.assert_allclose(p1, p2, rtol=0, atol=2e-6 * float(np.abs(p2).max()))
    np.testing.assert_allclose(r1, r2, rtol=0, atol=2e-6 * float(np.abs(r2).max()) * 4)


def test_filter_window_is_even():
    for n in (36, 37, 256, 301):
        w = O.filter_fill_plain(5, 0.0, n)
        assert np.array_equal(w, w[(-np.arange(n)) % n])
