"""Python mirror of the ctas reconstruction interface (src/common/ct.h).

``Filter``, ``Contrast`` and ``CTrec`` keep the reference's names, argument
meanings and error behaviour (a ``CtasError`` where the reference throws
``CtasErr``); the work is done by the CUDA library through the C ABI.  Arrays
are numpy float32 (host) or torch CUDA tensors (device forms).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CtasError, Opts, check, load

__all__ = ["Filter", "Contrast", "CTrec", "Batch", "CtasError", "padded_width", "angle_table",
           "rec_cof", "arc_rad", "probe_smem_gather", "probe_l2_read", "tile_shape"]


def probe_smem_gather(device: int = -1):
    """Measured shared-memory gather bandwidth (bytes/s) of the device."""
    bw, sec = C.c_double(), C.c_double()
    check(load().ctas_probe_smem_gather(device, C.byref(bw), C.byref(sec)))
    return bw.value


def probe_l2_read(device: int = -1):
    """Measured L2 read bandwidth (bytes/s) of the device."""
    bw, sec = C.c_double(), C.c_double()
    check(load().ctas_probe_l2_read(device, C.byref(bw), C.byref(sec)))
    return bw.value


def tile_shape(tile: int):
    """(rows, cols, window samples) of a staged backprojection tile id."""
    r, c, b = C.c_int32(), C.c_int32(), C.c_int32()
    check(load().ctas_fbp_tile_shape(int(tile), C.byref(r), C.byref(c), C.byref(b)))
    return r.value, c.value, b.value


class Contrast:
    """Contrast (src/common/physical.world.h:18-45)."""
    ABS, REF, PHS, FLT = 0, 1, 2, 3

    def __init__(self, cn=FLT):
        if isinstance(cn, str):
            v = C.c_int32()
            check(load().ctas_contrast_from_name(cn.encode(), C.byref(v)))
            cn = v.value
        if isinstance(cn, Contrast):
            cn = cn.contrast()
        if cn not in (0, 1, 2, 3):
            raise CtasError(_lib.E_ARG, f"unknown contrast {cn}")
        self._c = int(cn)

    def contrast(self) -> int:
        return self._c

    def name(self) -> str:
        return load().ctas_contrast_name(self._c).decode()

    def __eq__(self, o):
        return isinstance(o, Contrast) and o._c == self._c

    def __int__(self):
        return self._c


class Filter:
    """Filter (src/common/ct.h:87-162)."""
    NONE, RAMP, BARLETT, WELCH, PARZEN, HANN, HAMMING = 0, 1, 2, 3, 4, 5, 6
    BLACKMAN, LANCKZOS, KAISER, GAUSS = 7, 8, 9, 10
    SHEPP_LOGAN, COSINE = 100, 101  # extensions

    def __init__(self, tp=RAMP, param: float = 0.0):
        if isinstance(tp, str):
            v = C.c_int32()
            check(load().ctas_filter_from_name(tp.encode(), C.byref(v)))
            tp = v.value
        check(load().ctas_filter_check(int(tp), float(param)))
        self._t = int(tp)
        self._p = float(param)

    @classmethod
    def parse(cls, spec: str) -> "Filter":
        """_conversion(Filter*, string): "NAME[:float]" (lct.cpp:236-248)."""
        t, p = C.c_int32(), C.c_float()
        check(load().ctas_filter_parse(spec.encode(), C.byref(t), C.byref(p)))
        return cls(t.value, p.value)

    def filter(self) -> int:
        return self._t

    def param(self) -> float:
        return self._p

    def name(self) -> str:
        return load().ctas_filter_name(self._t).decode()

    def fill(self, pixels: int) -> np.ndarray:
        """Filter::fill (lct.cpp:122-209)."""
        out = np.zeros(pixels, np.float32)
        check(load().ctas_filter_fill(self._t, self._p, pixels, out.ctypes.data))
        return out

    def __eq__(self, o):  # ct.h:172-175 compares the type only
        return isinstance(o, Filter) and o._t == self._t


def tile_count() -> int:
    """Number of staged backprojection tile ids (valid ``tile`` values are
    0 .. tile_count()-1; -1 autotunes)."""
    return int(load().ctas_fbp_tile_count())


def padded_width(W: int) -> int:
    return int(load().ctas_fbp_padded_width(W))


def arc_rad(anarc: float, points: int) -> float:
    return float(load().ctas_fbp_arc(anarc, points))


def angle_table(arc_deg: float, N: int) -> np.ndarray:
    t = np.zeros(2 * N, np.float32)
    check(load().ctas_fbp_angle_table(arc_deg, N, t.ctypes.data))
    return t


def window(W: int, contrast, ftype, fparam: float = 0.0, pad: int = 0) -> np.ndarray:
    P = pad or padded_width(W)
    g = np.zeros(P, np.float32)
    check(load().ctas_fbp_window(W, int(Contrast(contrast)), int(ftype), fparam, pad,
                                 g.ctypes.data))
    return g


def rec_cof(pixel_size: float = 0.0, lam: float = 0.0) -> float:
    return float(load().ctas_fbp_rec_cof(pixel_size, lam))


def _f32(a: np.ndarray, shape: Sequence[int], what: str) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous:
        raise CtasError(_lib.E_ARG, f"{what} must be a C-contiguous float32 numpy array")
    if tuple(a.shape) != tuple(shape):
        raise CtasError(_lib.E_SHAPE, f"Wrong {what} shape {a.shape} where {tuple(shape)} "
                                      "is expected.")
    return a


def _dev_ptr(t, shape, what):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
            and t.is_contiguous()):
        raise CtasError(_lib.E_ARG, f"{what} must be a contiguous float32 CUDA tensor")
    if tuple(t.shape) != tuple(shape):
        raise CtasError(_lib.E_SHAPE, f"Wrong {what} shape {tuple(t.shape)} where "
                                      f"{tuple(shape)} is expected.")
    return C.c_void_p(t.data_ptr())


class CTrec:
    """CT reconstruction object (src/common/ct.h:235-298) on a CUDA device.

    ``CTrec(sinoshape, contrast, arc=180, filter=Filter())``; extensions are
    keyword-only: ``pad`` (FFT length), ``store`` (0 f32 / 1 f16 / 2 bf16),
    ``angles`` (radians), ``interp`` (0 reference truncation / 1 linear),
    ``no_writeback``, ``chunk_slices``, ``device``, ``checked`` (bounds-checked
    staged kernel, a test aid), ``tile`` (staged kernel tile id, -1 autotune),
    ``out_shape``/``out_pixel``/``out_shift`` (output geometry), ``ring_box``
    (ring-artefact filter half width, the ct tool's -R), ``index_rule``
    ("ctcl": the index expression rounded as ct.cl:36-37 writes it, the
    reference's OpenCL path; "shipped": as the reference's -ffast-math build
    rounds lct.cpp:711-712, its CPU path as built), ``flags`` (further
    CTAS_FLAG_* bits of ctas_fbp.h, e.g. test aids).
    """

    def __init__(self, sinoshape, cn=Contrast.FLT, arc: float = 180.0,
                 ft: Optional[Filter] = None, *, pad: int = 0, store: int = 0,
                 angles=None, interp: int = 0, no_writeback: bool = False,
                 chunk_slices: int = 0, device: int = -1, checked: bool = False,
                 tile: int = -1, out_shape=None, out_pixel: float = 0.0,
                 out_shift=(0.0, 0.0), ring_box: int = 0, index_rule: str = "ctcl",
                 flags: int = 0, _handle=None):
        self._h = None
        if index_rule not in ("ctcl", "shipped"):
            raise CtasError(_lib.E_ARG, f"unknown index rule {index_rule!r}")
        L = load()
        N, W = int(sinoshape[0]), int(sinoshape[1])
        self.ish = (N, W)
        if _handle is not None:
            self._h = _handle
        else:
            ft = ft or Filter()
            o = Opts()
            o.struct_size = C.sizeof(Opts)
            o.interp = interp
            o.pad = pad
            o.store = store
            o.device = device
            o.flags = ((_lib.FLAG_NO_WRITEBACK if no_writeback else 0) |
                       (_lib.FLAG_CHECKED if checked else 0) |
                       (_lib.FLAG_SHIPPED_INDEX if index_rule == "shipped" else 0) | int(flags))
            o.chunk_slices = chunk_slices
            o.tile = tile
            if out_shape is not None:
                o.out_rows, o.out_cols = int(out_shape[0]), int(out_shape[1])
            o.out_pixel = out_pixel
            o.ring_box = ring_box
            o.out_shift_row, o.out_shift_col = float(out_shift[0]), float(out_shift[1])
            self._angles = None
            if angles is not None:
                self._angles = np.ascontiguousarray(angles, np.float64)
                if self._angles.shape != (N,):
                    raise CtasError(_lib.E_SHAPE, "angle list must hold one angle per projection")
                o.angles = self._angles.ctypes.data_as(C.POINTER(C.c_double))
            h = C.c_void_p()
            check(L.ctas_fbp_create(C.byref(h), N, W, int(Contrast(cn)), ft.filter(),
                                    ft.param(), arc, C.byref(o)))
            self._h = h
        r, c = C.c_int64(), C.c_int64()
        check(L.ctas_fbp_out_shape(self._h, C.byref(r), C.byref(c)))
        self.osh = (r.value, c.value)

    # CTrec(CTrec&) (lct.cpp:529-545)
    def clone(self) -> "CTrec":
        h = C.c_void_p()
        check(load().ctas_fbp_clone(self._h, C.byref(h)))
        return CTrec(self.ish, _handle=h)

    def close(self):
        if self._h:
            load().ctas_fbp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def setPhysics(self, pixelSize: float = 0.0, lam: float = 0.0):
        check(load().ctas_fbp_set_physics(self._h, pixelSize, lam))

    def recShape(self, center: float = 0.0):
        r, c = C.c_int64(), C.c_int64()
        check(load().ctas_fbp_rec_shape(self._h, center, C.byref(r), C.byref(c)))
        return (r.value, c.value)

    # ---- host forms (synchronous), the reference's call shapes
    def sino(self, sinogram: np.ndarray) -> None:
        _f32(sinogram, self.ish, "sinogram")
        check(load().ctas_fbp_sino(self._h, sinogram.ctypes.data))

    def repeat(self, slice_: Optional[np.ndarray], center: float) -> np.ndarray:
        if slice_ is None:
            slice_ = np.empty(self.osh, np.float32)
        _f32(slice_, self.osh, "slice")
        check(load().ctas_fbp_repeat(self._h, slice_.ctypes.data, center))
        return slice_

    def reconstruct(self, sinogram: np.ndarray, slice_: Optional[np.ndarray] = None,
                    center: float = 0.0) -> np.ndarray:
        _f32(sinogram, self.ish, "sinogram")
        if slice_ is None:
            slice_ = np.empty(self.osh, np.float32)
        _f32(slice_, self.osh, "slice")
        check(load().ctas_fbp_reconstruct(self._h, sinogram.ctypes.data, slice_.ctypes.data,
                                          center))
        return slice_

    def reconstruct_stack(self, sinos: np.ndarray, slices: Optional[np.ndarray] = None,
                          center: float = 0.0) -> np.ndarray:
        S = sinos.shape[0]
        _f32(sinos, (S,) + self.ish, "sinogram stack")
        if slices is None:
            slices = np.empty((S,) + self.osh, np.float32)
        _f32(slices, (S,) + self.osh, "slice stack")
        check(load().ctas_fbp_reconstruct_stack(self._h, sinos.ctypes.data, slices.ctypes.data,
                                                S, center))
        return slices

    # ---- device forms (asynchronous on `stream`, torch CUDA tensors)
    @staticmethod
    def _stream(stream):
        if stream is None:
            import torch
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        return C.c_void_p(int(stream))

    def reconstruct_dev(self, sino, slice_, center: float = 0.0, stream=None):
        check(load().ctas_fbp_reconstruct_dev(self._h, _dev_ptr(sino, self.ish, "sinogram"),
                                              _dev_ptr(slice_, self.osh, "slice"), center,
                                              self._stream(stream)))
        return slice_

    def sino_dev(self, sino, filtered=None, stream=None):
        fp = _dev_ptr(filtered, self.ish, "filtered") if filtered is not None else None
        check(load().ctas_fbp_sino_dev(self._h, _dev_ptr(sino, self.ish, "sinogram"), fp,
                                       self._stream(stream)))

    def repeat_dev(self, slice_, center: float, stream=None):
        check(load().ctas_fbp_repeat_dev(self._h, _dev_ptr(slice_, self.osh, "slice"), center,
                                         self._stream(stream)))
        return slice_

    def repeat_multi_dev(self, centers, slices, stream=None):
        """Backprojects the last sino() at every centre into ``slices`` (a
        len(centers) x rows x cols CUDA tensor) in one launch (extension)."""
        cs = np.ascontiguousarray(np.atleast_1d(centers), np.float32)
        check(load().ctas_fbp_repeat_multi_dev(
            self._h, cs.ctypes.data_as(C.c_void_p), cs.size,
            _dev_ptr(slices, (cs.size,) + self.osh, "slice stack"), self._stream(stream)))
        return slices

    def reconstruct_stack_dev(self, sinos, slices, center: float = 0.0, stream=None):
        S = int(sinos.shape[0])
        check(load().ctas_fbp_reconstruct_stack_dev(
            self._h, _dev_ptr(sinos, (S,) + self.ish, "sinogram stack"),
            _dev_ptr(slices, (S,) + self.osh, "slice stack"), S, center, self._stream(stream)))
        return slices

    def synchronize(self):
        check(load().ctas_fbp_synchronize(self._h))

    def last_kernel(self) -> int:
        return int(load().ctas_fbp_last_kernel(self._h))

    def last_tile(self) -> int:
        return int(load().ctas_fbp_last_tile(self._h))

    def kernel_launches(self) -> int:
        return int(load().ctas_fbp_kernel_launches(self._h))

    def set_profiling(self, enable: bool = True):
        check(load().ctas_fbp_set_profiling(self._h, 1 if enable else 0))

    def profile_read(self, kind: int):
        """(total device ms, launches) of kernel kind 0 filter / 1 backprojection."""
        ms, n = C.c_double(), C.c_int64()
        check(load().ctas_fbp_profile_read(self._h, kind, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    # static one-shot form (ct.h:289-295)
    @staticmethod
    def reconstruct_once(sinogram, slice_=None, cn=Contrast.FLT, arc=180.0, ft=None,
                         center=0.0, pixelSize=0.0, lam=0.0, **kw):
        with CTrec(sinogram.shape, cn, arc, ft, **kw) as rec:
            rec.setPhysics(pixelSize, lam)
            return rec.reconstruct(sinogram, slice_, center)


class Batch:
    """Uneven batch of sinograms (extension): every (sinogram, slice) pair of
    torch CUDA tensors reconstructed by one graph launch.  ``jobs`` is a list
    of (sino [N, W], slice [W, W], centre)."""

    def __init__(self, jobs, cn=Contrast.PHS, arc: float = 180.0, ft: Optional[Filter] = None,
                 pixelSize: float = 0.0, lam: float = 0.0, *, pad: int = 0, tile: int = -1,
                 index_rule: str = "ctcl"):
        ft = ft or Filter()
        if index_rule not in ("ctcl", "shipped"):
            raise CtasError(_lib.E_ARG, f"unknown index rule {index_rule!r}")
        self._keep = [(s, o) for s, o, _ in jobs]
        arr = (_lib.Job * len(jobs))()
        for k, (s, o, c) in enumerate(jobs):
            N, W = int(s.shape[0]), int(s.shape[1])
            arr[k].n_angles, arr[k].width, arr[k].center = N, W, float(c)
            arr[k].sino_dev = _dev_ptr(s, (N, W), "sinogram").value
            arr[k].slice_dev = _dev_ptr(o, (W, W), "slice").value
        o = Opts()
        o.struct_size = C.sizeof(Opts)
        o.pad = pad
        o.device = -1
        o.tile = tile
        o.flags = _lib.FLAG_SHIPPED_INDEX if index_rule == "shipped" else 0
        h = C.c_void_p()
        check(load().ctas_fbp_batch_create(C.byref(h), arr, len(jobs), int(Contrast(cn)),
                                           ft.filter(), ft.param(), arc, pixelSize, lam,
                                           C.byref(o)))
        self._h = h

    def run(self, stream=None):
        check(load().ctas_fbp_batch_run(self._h, CTrec._stream(stream)))

    def run_loop(self, stream=None):
        check(load().ctas_fbp_batch_run_loop(self._h, CTrec._stream(stream)))

    def synchronize(self):
        check(load().ctas_fbp_batch_synchronize(self._h))

    def tile(self) -> int:
        return int(load().ctas_fbp_batch_tile(self._h))

    def close(self):
        if getattr(self, "_h", None):
            load().ctas_fbp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
