"""The oracle itself: pinned against the reference's own backprojection kernel
(ctas src/common/ct.cl, compiled for the host by oracle/Makefile) and the
committed golden fixtures, and against known answers for the filter stage."""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("N,W,c,arc", [(90, 64, 0.0, 180.0), (91, 65, 3.5, 180.0),
                                       (120, 96, -7.25, 360.0), (60, 48, 2.0, 0.5),
                                       (33, 32, -1.5, 180.0)])
def test_bp_oracle_matches_reference_kernel(N, W, c, arc):
    if not O.ref_available():
        pytest.skip("reference kernel not built here (reference sources absent)")
    rng = np.random.default_rng(N * 1000 + W)
    q = rng.standard_normal((N, W)).astype(np.float32)
    tab = O.angle_table(arc, N)
    a = O.bp_compat(q, tab, c, 1.0)
    b = O.ref_fbp(q, tab, c, 1.0, nthreads=2)
    assert np.array_equal(_bits(a), _bits(b))
    # physics coefficient path (coeff != 0)
    cof = O.rec_cof(1e-6, 1e-10)
    assert np.array_equal(_bits(O.bp_compat(q, tab, c, cof)), _bits(O.ref_fbp(q, tab, c, cof)))


def test_golden_fixtures_present():
    files = sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz")))
    assert len(files) >= 6


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz"))))
def test_oracle_matches_golden(path):
    z = np.load(path)
    tab = O.angle_table(float(z["arc"]), int(z["q"].shape[0]))
    assert np.array_equal(_bits(tab), _bits(z["tab"]))
    out = O.bp_compat(z["q"], tab, float(z["center"]), float(z["coeff"]))
    assert np.array_equal(_bits(out), _bits(z["slice"]))


def test_padded_width_rule():
    # lct.cpp:490
    assert [O.padded_width(w) for w in (2, 3, 100, 512, 513, 2048, 2560, 4096)] == \
        [4, 8, 256, 1024, 2048, 4096, 8192, 8192]


def test_mask_vectorised_matches_scalar():
    for W, c in ((64, 0.0), (65, 3.5), (64, -7.25)):
        m = O.mask(W, c)
        m2 = np.array([[O.in_mask(j, i, W, c) for i in range(W)] for j in range(W)])
        assert np.array_equal(m, m2)


def _ramlak(k):
    k = np.asarray(k, dtype=np.float64)
    out = np.zeros_like(k)
    out[k == 0] = 0.25
    odd = (k.astype(np.int64) % 2) != 0
    out[odd] = -1.0 / (k[odd] ** 2 * np.pi ** 2)
    return out


def test_filter_impulse_response_is_ramlak():
    # y = HC2R(R2HC(z) * G)/P with the RAMP window is (P/2W) * (z conv h_RamLak)
    N, W = 3, 100
    P = O.padded_width(W)
    G = O.filter_window(1, 0.0, P, W, O.PHS)
    x = np.zeros((N, W), np.float32)
    x[1, 37] = 1.0
    q = O.prepare_sino(x, P, O.PHS, G)
    np.testing.assert_allclose(q[1], P / (2 * W) * _ramlak(np.arange(W) - 37), atol=2e-8)
    assert np.abs(q[0]).max() == 0 and np.abs(q[2]).max() == 0


def test_filter_next_row_sample_quirk():
    # lct.cpp:580,584: the padded row also receives x[r+1][0] at zs+W
    N, W = 3, 100
    P = O.padded_width(W)
    G = O.filter_window(1, 0.0, P, W, O.PHS)
    x = np.zeros((N, W), np.float32)
    x[1, 0] = 1.0
    q = O.prepare_sino(x, P, O.PHS, G)
    np.testing.assert_allclose(q[0], P / (2 * W) * _ramlak(np.arange(W) - W), atol=2e-8)


@pytest.mark.parametrize("ft", [1, 3, 4, 5, 6, 7, 8, 9, 10, 100, 101])
def test_filter_matches_numpy_fft(ft):
    rng = np.random.default_rng(ft)
    N, W = 5, 100
    P = O.padded_width(W)
    zs = (P - W) // 2
    x = rng.random((N, W)).astype(np.float32)
    G = O.filter_window(ft, 1.5, P, W, O.PHS)
    assert np.array_equal(G[1:], G[1:][::-1])   # even window
    q = O.prepare_sino(x, P, O.PHS, G)
    ref = []
    for r in range(N):
        z = np.zeros(P)
        z[zs:zs + W] = x[r]
        z[zs + W] = x[r + 1, 0] if r + 1 < N else 0.0
        ref.append(np.fft.ifft(np.fft.fft(z) * G.astype(np.float64)).real[zs:zs + W])
    ref = np.array(ref)
    assert np.abs(q - ref).max() <= 1e-6 * np.abs(ref).max()


def test_window_values():
    # Hann window at the FFT bins (lct.cpp:175-176) against the closed form
    P, W = 256, 128
    G = O.filter_window(5, 0.0, P, W, O.PHS, fp64=True)
    R = O.filter_window(1, 0.0, P, W, O.PHS, fp64=True)
    m = np.minimum(np.arange(P), P - np.arange(P))
    f = m * 2.0 / P
    np.testing.assert_allclose(G, R * 0.5 * (1 + np.cos(np.pi * f)), rtol=1e-12, atol=1e-15)
    # REF contrast zeroes the DC bin (lct.cpp:507-508)
    assert O.filter_window(1, 0.0, P, W, O.REF)[0] == 0.0


def test_deabs():
    x = np.array([[2.0, 0.5, -1.0, 0.0]], np.float32)
    y = O.deabs(x)
    mina = np.float32(np.float64(2.0) / 1e6)
    np.testing.assert_array_equal(y, -np.log(np.maximum(x, mina)).astype(np.float32))
    with pytest.raises(ValueError):
        O.deabs(np.array([[-1.0, 0.0]], np.float32))


def test_ref_contrast_is_prefix_sum():
    rng = np.random.default_rng(5)
    N, W = 4, 50
    P = O.padded_width(W)
    x = rng.random((N, W)).astype(np.float32)
    Gp = O.filter_window(1, 0.0, P, W, O.REF)
    qp = O.prepare_sino(x, P, O.PHS, Gp)
    qr = O.prepare_sino(x, P, O.REF, Gp)
    np.testing.assert_allclose(qr, np.cumsum(qp.astype(np.float64), axis=1), rtol=1e-5, atol=1e-6)


def test_angle_table_float_semantics():
    N = 1800
    tab = O.angle_table(180.0, N)
    arc = np.float32(np.float64(np.float32(180.0)) * (np.pi / 180))
    th = np.arange(N, dtype=np.float32) * arc / np.float32(N)
    # sinf/cosf of the float angles: within one ulp of the correctly rounded value
    ulp = np.spacing(np.abs(tab[1::2]))
    assert (np.abs(tab[1::2] - np.cos(th.astype(np.float64))) <= ulp).all()
    ulp = np.spacing(np.abs(tab[0::2]))
    assert (np.abs(tab[0::2] - np.sin(th.astype(np.float64))) <= ulp).all()
    assert (tab[0::2] >= 0).all()


def test_linear_oracle_reconstructs_phantom():
    from ctas_b200 import phantom as ph
    W, N, c = 96, 240, 2.5
    el = ph.random_ellipses(7, 4, W, axes=(6, 20))
    s = ph.sinogram(el, N, W, center=c)
    P = O.padded_width(W)
    G = O.filter_window(5, 0.0, P, W, O.PHS, fp64=True)
    qd = O.prepare_sino(s, P, O.PHS, G, fp64=True)
    lin = O.bp_linear(qd, O.angle_table_f64(180.0, N), c, np.pi * 2 * W / P)
    trunc = O.bp_compat(qd, O.angle_table(180.0, N), c, np.pi * 2 * W / P)
    img = ph.image(el, W, c)
    m = O.mask(W, c)
    e_lin = np.abs(lin - img)[m].mean()
    e_trunc = np.abs(trunc - img)[m].mean()
    assert e_lin < 0.1 and e_trunc < 0.12
