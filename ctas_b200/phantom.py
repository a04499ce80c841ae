"""Seeded analytic phantoms and their exact parallel-beam projections (FP64).

The geometry is the one the reference's backprojector assumes
(ctas src/common/lct.cpp:711-713): for projection angle th the pixel
(row j, column i) of a W x W slice lands on detector coordinate
    t = (hp + c) + sin(th) * (j - hp - c) + cos(th) * (i - hp),   hp = W // 2,
and detector sample k covers t in [k, k + 1).  Sample k of a sinogram made
here is the line integral at the sample centre t = k + 0.5, so an object at
object coordinates (x, y) = (i - hp, j - hp - c) reconstructs at pixel (j, i).

Ellipses: centre (x0, y0), semi-axes (a, b), orientation phi, density rho.
The projection along direction n = (cos th, sin th) at offset u from the
ellipse centre is 2 rho a b sqrt(r^2 - u^2) / r^2 with
r^2 = a^2 (n . e_a)^2 + b^2 (n . e_b)^2 (zero for |u| >= r).
"""
from __future__ import annotations

import numpy as np


def random_ellipses(seed: int, n: int, W: int, axes=(5.0, 120.0), rho=(0.1, 1.0),
                    scale: float = 1.0) -> np.ndarray:
    """n random ellipses inside a W x W field: rows (x0, y0, a, b, phi, rho).

    Semi-axes U(axes)*scale, orientation U(0, pi), density U(rho); centres are
    drawn so that each ellipse lies inside the disc the reference reconstructs.
    """
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 6))
    R = 0.5 * W - 2.0
    for k in range(n):
        a, b = rng.uniform(axes[0], axes[1], 2) * scale
        a, b = min(a, 0.45 * R), min(b, 0.45 * R)
        rmax = max(R - max(a, b), 0.0)
        rr = rmax * np.sqrt(rng.uniform(0, 1))
        ang = rng.uniform(0, 2 * np.pi)
        out[k] = (rr * np.cos(ang), rr * np.sin(ang), a, b, rng.uniform(0, np.pi),
                  rng.uniform(*rho))
    return out


def sinogram(ellipses: np.ndarray, N: int, W: int, center: float = 0.0,
             arc_deg: float = 180.0, angles=None, dtype=np.float32) -> np.ndarray:
    """Exact projections of the ellipses, N x W, angles i*arc/N (or `angles`)."""
    th = (np.arange(N) * (np.deg2rad(arc_deg) / N)) if angles is None else np.asarray(angles)
    cs, sn = np.cos(th)[:, None], np.sin(th)[:, None]
    hp = W // 2
    u = (np.arange(W) + 0.5 - (hp + center))[None, :]
    out = np.zeros((N, W))
    for x0, y0, a, b, phi, rho in ellipses:
        if a <= 0 or b <= 0:
            continue
        ca, sa = np.cos(phi), np.sin(phi)
        na = cs * ca + sn * sa          # n . e_a
        nb = -cs * sa + sn * ca         # n . e_b
        r2 = a * a * na * na + b * b * nb * nb
        d = u - (cs * x0 + sn * y0)
        q = r2 - d * d
        out += np.where(q > 0, 2.0 * rho * a * b * np.sqrt(np.maximum(q, 0)) / r2, 0.0)
    return out.astype(dtype)


def image(ellipses: np.ndarray, W: int, center: float = 0.0) -> np.ndarray:
    """The phantom sampled at pixel centres of the W x W slice grid."""
    hp = W // 2
    j, i = np.mgrid[0:W, 0:W]
    x = i - hp + 0.0
    y = j - hp - center + 0.0
    img = np.zeros((W, W))
    for x0, y0, a, b, phi, rho in ellipses:
        if a <= 0 or b <= 0:
            continue
        ca, sa = np.cos(phi), np.sin(phi)
        xr = (x - x0) * ca + (y - y0) * sa
        yr = -(x - x0) * sa + (y - y0) * ca
        img += np.where((xr / a) ** 2 + (yr / b) ** 2 <= 1.0, rho, 0.0)
    return img


def poisson_log(p: np.ndarray, photons: float, seed: int) -> np.ndarray:
    """Line integrals with Poisson noise: -log(Poisson(I0 e^-p)/I0), with zero
    counts clamped the way deAbs clamps (physical.world.cpp:89-98)."""
    rng = np.random.default_rng(seed)
    counts = rng.poisson(photons * np.exp(-p.astype(np.float64))).astype(np.float64)
    tr = counts / photons
    mx = tr.max()
    tr = np.maximum(tr, mx / 1e6)
    return (-np.log(tr)).astype(np.float32)


def random_ellipsoids(seed: int, n: int, W: int, depth: int, rho=(0.05, 0.5),
                      axes=(0.05, 0.35)) -> np.ndarray:
    """n random ellipsoids in a W x W x depth volume, each with one axis along
    z: rows (x0, y0, z0, a, b, c, phi, rho); semi-axes U(axes) * W/2 in x, y and
    U(axes) * depth/2 in z."""
    rng = np.random.default_rng(seed)
    R = 0.5 * W - 2.0
    out = np.zeros((n, 8))
    for k in range(n):
        a, b = rng.uniform(*axes, 2) * R
        c = rng.uniform(*axes) * depth / 2 + 1.0
        rmax = max(R - max(a, b), 0.0)
        rr = rmax * np.sqrt(rng.uniform(0, 1))
        ang = rng.uniform(0, 2 * np.pi)
        out[k] = (rr * np.cos(ang), rr * np.sin(ang), rng.uniform(0, depth), a, b, c,
                  rng.uniform(0, np.pi), rng.uniform(*rho))
    return out


def ellipsoid_sections(ellipsoids: np.ndarray, z: float) -> np.ndarray:
    """The ellipses cut by the plane at height z (zero-size rows where the
    plane misses an ellipsoid)."""
    x0, y0, z0, a, b, c, phi, rho = ellipsoids.T
    f = 1.0 - ((z - z0) / c) ** 2
    s = np.sqrt(np.clip(f, 0.0, None))
    return np.stack([x0, y0, a * s, b * s, phi, np.where(f > 0, rho, 0.0)], axis=1)


def sinogram_dev(ellipses_per_slice: np.ndarray, N: int, W: int, center: float = 0.0,
                 arc_deg: float = 180.0, stream=None):
    """Exact projections on the device: ellipses_per_slice is S x E x 6;
    returns a torch float32 CUDA tensor S x N x W."""
    import ctypes as C

    import torch

    from . import _lib
    L = _lib.load()
    fn = L.ctas_phantom_sinogram_dev
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_void_p,
                   C.c_double, C.c_void_p, C.c_void_p]
    el = torch.as_tensor(np.ascontiguousarray(ellipses_per_slice, np.float64), device="cuda")
    S, E = int(el.shape[0]), int(el.shape[1])
    th = torch.as_tensor(np.arange(N) * (np.deg2rad(arc_deg) / N), device="cuda",
                         dtype=torch.float64)
    out = torch.empty((S, N, W), device="cuda", dtype=torch.float32)
    st = torch.cuda.current_stream().cuda_stream if stream is None else int(stream)
    _lib.check(fn(el.data_ptr(), E, S, N, W, th.data_ptr(), center, out.data_ptr(), st))
    return out


def angles_dev(N: int, arc_deg: float = 180.0):
    """Projection angles i * arc / N (radians) as an FP64 CUDA tensor."""
    import torch
    return torch.as_tensor(np.arange(N) * (np.deg2rad(arc_deg) / N), device="cuda",
                           dtype=torch.float64)


def project_image_dev(img, N: int, center: float = 0.0, arc_deg: float = 180.0, out=None,
                      radius=None, step: float = 0.5, stream=None):
    """Ray-marched line integrals of images (torch float32 CUDA, S x W x W, the
    slice grid of a reconstruction with this centre) added to `out` (S x N x W,
    zeros if None); rays are sampled every `step` px along their chord of the
    disc of `radius` (default W/2 - 1) around the axis."""
    import torch

    from . import _lib
    if img.dim() == 2:
        img = img[None]
    img = img.contiguous().float()
    S, W = int(img.shape[0]), int(img.shape[-1])
    if out is None:
        out = torch.zeros((S, N, W), device="cuda", dtype=torch.float32)
    th = angles_dev(N, arc_deg)
    r = float(W / 2 - 1) if radius is None else float(radius)
    st = torch.cuda.current_stream().cuda_stream if stream is None else int(stream)
    _lib.check(_lib.load().ctas_phantom_project_image_dev(img.data_ptr(), S, N, W, th.data_ptr(),
                                                          float(center), r, float(step),
                                                          out.data_ptr(), st))
    return out


def grf_texture_dev(seed: int, W: int, S: int = 1, std: float = 0.05, corr_px: float = 8.0,
                    center: float = 0.0, radius=None):
    """Band-limited Gaussian random field: white noise low-passed by a Gaussian
    of correlation length corr_px, scaled to standard deviation `std` and
    confined to the disc of `radius` (default W/2 - 2 - |center|) around the
    rotation axis, pixel (W/2 + center, W/2) of the slice grid.  torch float32
    CUDA, S x W x W."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed))
    noise = torch.randn((S, W, W), device="cuda", generator=g)
    f = torch.fft.fftfreq(W, device="cuda")
    k2 = f[:, None] ** 2 + f[None, :] ** 2
    lp = torch.exp(-2.0 * (np.pi * corr_px) ** 2 * k2)
    field = torch.fft.ifft2(torch.fft.fft2(noise) * lp).real
    field = field / field.std(dim=(1, 2), keepdim=True) * std
    hp = W // 2
    j = torch.arange(W, device="cuda", dtype=torch.float32)[:, None] - hp - float(center)
    i = torch.arange(W, device="cuda", dtype=torch.float32)[None, :] - hp
    r = float(W / 2 - 2 - abs(center)) if radius is None else float(radius)
    return (field * ((i * i + j * j) <= r * r)).float().contiguous()


def image_dev(ellipses: np.ndarray, W: int, center: float = 0.0):
    """image() on the device (FP64 evaluation, float32 result): the ellipses
    sampled at the pixel centres of the W x W slice grid."""
    import torch
    hp = W // 2
    j = torch.arange(W, device="cuda", dtype=torch.float64)[:, None]
    i = torch.arange(W, device="cuda", dtype=torch.float64)[None, :]
    x, y = i - hp, j - hp - center
    img = torch.zeros((W, W), device="cuda", dtype=torch.float64)
    for x0, y0, a, b, phi, rho in ellipses:
        if a <= 0 or b <= 0:
            continue
        ca, sa = float(np.cos(phi)), float(np.sin(phi))
        xr = (x - x0) * ca + (y - y0) * sa
        yr = -(x - x0) * sa + (y - y0) * ca
        img += ((xr / a) ** 2 + (yr / b) ** 2 <= 1.0).double() * float(rho)
    return img.float()
