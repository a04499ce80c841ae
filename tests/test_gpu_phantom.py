"""GPU tests of the synthetic-input generator: the ray-marched image
projector against closed-form line integrals, and the band-limited texture."""
import numpy as np
import pytest

from ctas_b200 import phantom as ph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("center", [0.0, 3.5, -12.25])
def test_projector_matches_gaussian_blob_integrals(center):
    """A Gaussian blob of width sigma at object point (x0, y0) projects to
    sqrt(2 pi) sigma exp(-(u - x0 cos th - y0 sin th)^2 / (2 sigma^2))."""
    import torch
    W, N, sig, x0, y0 = 256, 90, 12.0, 20.0, -15.0
    hp = W // 2
    j = torch.arange(W, device="cuda", dtype=torch.float64)[:, None]
    i = torch.arange(W, device="cuda", dtype=torch.float64)[None, :]
    x, y = i - hp, j - hp - center
    img = torch.exp(-((x - x0) ** 2 + (y - y0) ** 2) / (2 * sig * sig)).float()
    got = ph.project_image_dev(img, N, center=center)[0].cpu().numpy().astype(np.float64)
    th = np.arange(N) * (np.pi / N)
    u = np.arange(W) + 0.5 - (hp + center)
    want = np.sqrt(2 * np.pi) * sig * np.exp(
        -(u[None, :] - (x0 * np.cos(th) + y0 * np.sin(th))[:, None]) ** 2 / (2 * sig * sig))
    assert np.abs(got - want).max() <= 3e-3 * want.max()


def test_projector_adds_into_out_and_is_linear():
    import torch
    W, N = 128, 40
    a = ph.grf_texture_dev(1, W, std=0.05)
    b = ph.grf_texture_dev(2, W, std=0.05)
    pa = ph.project_image_dev(a, N)
    pab = ph.project_image_dev(b, N, out=pa.clone())
    pb = ph.project_image_dev(b, N)
    assert float((pab - (pa + pb)).abs().max()) <= 1e-5 * float(pab.abs().max())


def test_texture_is_band_limited_and_confined():
    import torch
    W = 256
    t = ph.grf_texture_dev(7, W, S=2, std=0.05, corr_px=8.0, center=6.0)
    assert t.shape == (2, W, W)
    inside = t[t != 0]
    assert abs(float(inside.std()) - 0.05) < 0.01
    # confined to the disc of radius W/2 - 2 - |c| around pixel (W/2 + c, W/2)
    j = torch.arange(W, device="cuda")[:, None] - W // 2 - 6.0
    i = torch.arange(W, device="cuda")[None, :] - W // 2
    outside = (i * i + j * j) > (W / 2 - 8) ** 2
    assert float(t[:, outside].abs().max()) == 0.0
    # neighbouring pixels are strongly correlated (band-limited)
    c = torch.corrcoef(torch.stack([t[0, 100:150, 100:150].flatten(),
                                    t[0, 100:150, 101:151].flatten()]))[0, 1]
    assert float(c) > 0.9


def test_image_dev_matches_host_image():
    ell = ph.random_ellipses(3, 6, 128, axes=(5.0, 40.0))
    host = ph.image(ell, 128, center=2.5).astype(np.float32)
    dev = ph.image_dev(ell, 128, center=2.5).cpu().numpy()
    # identical up to pixels on an ellipse boundary (last-bit differences of
    # the inside test)
    assert np.mean(dev != host) < 1e-3
