"""Rotation-axis search (the ``ctas axis`` tool) on the GPU path.

Python face of include/ctas_axis.h, mirroring the reference's
``AverageGradient`` class and ``raxis()`` functions (ctas
src/common/lct.cpp:792-1297, src/common/ct.h:327-329).  Axis positions are
absolute detector coordinates; the ``axis`` tool prints
``raxis(...) - 0.5 * (width - 1)`` (src/executables/axis.cpp:126).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CtasError, check, load


def _host(a, what: str) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float32)
    if a.ndim != 2:
        raise CtasError(-2, f"{what} must be two-dimensional")
    return a


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class AverageGradient:
    """``AverageGradient(sino, anarc=180)`` (lct.cpp:800-915): filters a copy of
    the absorption sinogram once; ``apply(axis_r)`` reconstructs about each
    axis position and returns the mean gradient magnitude of the smoothed,
    cropped slice.  ``apply`` takes one position or a sequence (evaluated as
    batched multi-centre backprojections)."""

    def __init__(self, sino, anarc: float = 180.0, *, device: int = -1,
                 index_rule: str = "ctcl"):
        self._h = None
        s = _host(sino, "sinogram")
        h = C.c_void_p()
        flags = {"ctcl": 0, "shipped": _lib.FLAG_SHIPPED_INDEX}[index_rule]
        check(load().ctas_ag_create_flags(C.byref(h), _fp(s), s.shape[0], s.shape[1],
                                          float(anarc), int(device), flags))
        self._h = h
        self.ish = s.shape

    def apply(self, axis_r):
        scalar = np.ndim(axis_r) == 0
        ax = np.ascontiguousarray(np.atleast_1d(axis_r), np.float32)
        out = np.zeros(ax.shape, np.float32)
        check(load().ctas_ag_apply(self._h, _fp(ax), ax.size, _fp(out)))
        return out[0] if scalar else out

    @property
    def sigma(self) -> float:
        s = C.c_float()
        check(load().ctas_ag_sigma(self._h, C.byref(s), None))
        return s.value

    @property
    def taps(self) -> int:
        k = C.c_int32()
        check(load().ctas_ag_sigma(self._h, None, C.byref(k)))
        return k.value

    def close(self):
        if self._h:
            load().ctas_ag_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def raxis(sino, anarc: float, max_dev: float, algo: int = 0, *, device: int = -1,
          return_trials: bool = False):
    """``raxis(sino, anarc, maxDev, algo)`` (lct.cpp:1137-1212): absolute
    rotation-axis position of an absorption sinogram.  ``algo`` 0: projection
    pair only; 1: average-gradient search from the centre; 2: from the pair
    estimate; 3: from a threshold estimate."""
    s = _host(sino, "sinogram")
    ax = C.c_float()
    n = C.c_int64()
    check(load().ctas_raxis(_fp(s), s.shape[0], s.shape[1], float(anarc), float(max_dev),
                            int(algo), int(device), C.byref(ax), C.byref(n)))
    return (ax.value, n.value) if return_trials else ax.value


def raxis_pair(proj0, proj180, max_dev: float, *, device: int = -1) -> float:
    """``raxis(proj0, proj180, maxDev)`` (lct.cpp:1217-1297): rotation axis from
    two opposite projections (rows x width each)."""
    p0 = _host(proj0, "proj0")
    p1 = _host(proj180, "proj180")
    if p0.shape != p1.shape:
        raise CtasError(-2, "Different shapes of input projections")
    ax = C.c_float()
    check(load().ctas_raxis_pair(_fp(p0), _fp(p1), p0.shape[0], p0.shape[1], float(max_dev),
                                 int(device), C.byref(ax)))
    return ax.value
