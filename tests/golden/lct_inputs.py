"""Seeded inputs of the lct_*.npz fixtures, regenerated by the tests.

Each input is an analytic phantom projection (ctas_b200.phantom, FP64) or a
seeded random array, rounded to a multiple of 2^-12 before it is stored as
float32, so that last-bit differences of the host's FP64 maths libraries
cannot change it; the fixture stores its SHA-256 and the tests check it.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from ctas_b200 import phantom as ph  # noqa: E402

Q = 4096.0


def quantise(x: np.ndarray) -> np.ndarray:
    return (np.round(np.asarray(x, np.float64) * Q) / Q).astype(np.float32)


def sha(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()


def ellipse_sino(seed: int, N: int, W: int, center: float, arc: float = 180.0, n: int = 10,
                 axes=(5.0, 120.0), rho=(0.1, 1.0), photons: float = 0.0) -> np.ndarray:
    """Projections of n seeded random ellipses (the configs' phantom family),
    N projections evenly spaced over `arc` degrees; with photons > 0 the
    Poisson-noised -log(counts / photons) of exp(-p)."""
    el = ph.random_ellipses(seed, n, W, axes=axes, rho=rho)
    p = ph.sinogram(el, N, W, center=center, arc_deg=arc, dtype=np.float64)
    if photons > 0:
        rng = np.random.default_rng(seed + 7)
        cnt = rng.poisson(photons * np.exp(-p)).astype(np.float64)
        p = -np.log(np.maximum(cnt, 1.0) / photons)
    return quantise(p)


def transmission(seed: int, N: int, W: int, center: float) -> np.ndarray:
    """exp(-p) of an ellipse phantom with a few zero and negative samples (the
    inputs deAbs clamps, physical.world.cpp:88-100)."""
    p = ellipse_sino(seed, N, W, center, n=6, axes=(5.0, W / 5.0))
    t = np.exp(-2.0 * p / max(float(p.max()), 1e-6))
    t[N // 3, W // 4:W // 4 + 7] = 0.0
    t[N // 2, W // 2] = -0.25
    return quantise(t)


def normal(seed: int, N: int, W: int) -> np.ndarray:
    return quantise(np.random.default_rng(seed).standard_normal((N, W)))
