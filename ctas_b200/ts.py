"""Tomosynthesis step ``ts_add`` (the ``ctas ts`` tool) on the GPU path.

Python face of include/ctas_ts.h, mirroring ts_add(projection, result, filter,
center, contrast, angle, plane) (ctas src/common/lct.cpp:731-787).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import FLAG_NO_WRITEBACK, CtasError, check, load
from .ct import Contrast, Filter, _dev_ptr


class TS:
    """``TS((rows, pixels), filter, contrast)``: prepared ts_add for projection
    images of that shape.  ``add(projection, result, center, angle, plane)``
    filters ``projection`` in place (as the reference does) and accumulates
    ``result``; ``add_dev`` / ``add_batch_dev`` take CUDA tensors."""

    def __init__(self, shape, ft: Filter | None = None, cn=Contrast.PHS, *, device: int = -1):
        ft = ft or Filter()
        self._h = None
        self.shape = (int(shape[0]), int(shape[1]))
        h = C.c_void_p()
        check(load().ctas_ts_create(C.byref(h), self.shape[0], self.shape[1], ft.filter(),
                                    ft.param(), int(Contrast(cn)), int(device)))
        self._h = h

    def add(self, projection: np.ndarray, result: np.ndarray, center: float, angle: float,
            plane: int, *, writeback: bool = True):
        for a, what in ((projection, "projection"), (result, "result")):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous
                    and a.shape == self.shape):
                raise CtasError(-2, f"{what} must be a contiguous float32 array of shape "
                                    f"{self.shape}")
        check(load().ctas_ts_add(self._h, projection.ctypes.data_as(C.c_void_p),
                                 result.ctypes.data_as(C.c_void_p), float(center), float(angle),
                                 int(plane), 0 if writeback else FLAG_NO_WRITEBACK))
        return result

    def add_dev(self, projection, result, center: float, angle: float, plane: int, *,
                writeback: bool = True, stream=None):
        check(load().ctas_ts_add_dev(self._h, _dev_ptr(projection, self.shape, "projection"),
                                     _dev_ptr(result, self.shape, "result"), float(center),
                                     float(angle), int(plane),
                                     0 if writeback else FLAG_NO_WRITEBACK,
                                     C.c_void_p(stream) if stream else None))
        return result

    def add_batch_dev(self, projections, angles, result, center: float, plane: int, *,
                      writeback: bool = True, stream=None):
        ang = np.ascontiguousarray(np.atleast_1d(angles), np.float32)
        check(load().ctas_ts_add_batch_dev(
            self._h, _dev_ptr(projections, (ang.size,) + self.shape, "projections"),
            ang.ctypes.data_as(C.c_void_p), ang.size, _dev_ptr(result, self.shape, "result"),
            float(center), int(plane), 0 if writeback else FLAG_NO_WRITEBACK,
            C.c_void_p(stream) if stream else None))
        return result

    def close(self):
        if self._h:
            load().ctas_ts_destroy(self._h)
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
