"""CPU oracle for the ctas FBP hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference
legs of bench.py may import this package.  It wraps two host libraries built by
``oracle/Makefile``:

* ``_build/liboracle.so`` -- fbp_oracle.c, the C restatement of the reference
  algorithm (ctas src/common/lct.cpp:122-209, 280-291, 470-517, 558-597,
  688-729 and src/common/physical.world.cpp:88-100) in FP32-compatible and
  FP64 forms;
* ``_ref/libctcl_ref.so`` -- the reference's own backprojection kernel
  (ctas src/common/ct.cl:5-44) compiled for the host.  It exists only where the
  reference sources were present when the oracle was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libctcl_ref.so")

# Contrast::Cntype (src/common/physical.world.h:22-27)
ABS, REF, PHS, FLT = 0, 1, 2, 3
# Filter::Ftype (src/common/ct.h:92-132) + two extension windows
FILTERS = {"NONE": 0, "RAMP": 1, "BARLETT": 2, "WELCH": 3, "PARZEN": 4,
           "HANN": 5, "HAMMING": 6, "BLACKMAN": 7, "LANCKZOS": 8,
           "KAISER": 9, "GAUSS": 10, "SHEPP_LOGAN": 100, "COSINE": 101}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_lib = None
_ref = None


def build(with_ref: bool | None = None) -> None:
    """Build the oracle (and, when the reference tree exists, oracle/_ref)."""
    targets = ["all"]
    src = os.environ.get("CTAS_REFERENCE_SRC", "/root/reference/src/common")
    if with_ref is None:
        with_ref = os.path.exists(os.path.join(src, "ct.cl"))
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets, f"REFERENCE_SRC={src}"],
                   check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_ref=False)
        L = C.CDLL(LIB_PATH)
        L.orc_padded_width.restype = C.c_int64
        L.orc_padded_width.argtypes = [C.c_int64]
        L.orc_filter_fill.restype = C.c_int
        L.orc_filter_fill.argtypes = [C.c_int, C.c_float, C.c_int64, C.c_int64,
                                      C.c_int, C.c_void_p, C.c_void_p]
        L.orc_arc.restype = C.c_float
        L.orc_arc.argtypes = [C.c_float, C.c_int64]
        L.orc_angle_table.argtypes = [C.c_float, C.c_int64, _f32p]
        L.orc_angle_table_f64.argtypes = [C.c_double, C.c_int64, _f64p]
        L.orc_angle_table_list.argtypes = [_f64p, C.c_int64, _f32p]
        L.orc_rec_cof.restype = C.c_float
        L.orc_rec_cof.argtypes = [C.c_float, C.c_float]
        L.orc_deabs.restype = C.c_int
        L.orc_deabs.argtypes = [_f32p, C.c_int64]
        L.orc_prepare_sino.restype = C.c_int
        L.orc_prepare_sino.argtypes = [_f32p, C.c_int64, C.c_int64, C.c_int64,
                                       C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        L.orc_in_mask.restype = C.c_int
        L.orc_in_mask.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_float]
        L.orc_bp_compat.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                    _f32p, C.c_float, C.c_float, C.c_int64,
                                    C.c_int64, C.c_void_p, C.c_void_p]
        L.orc_bp_linear.argtypes = [_f64p, C.c_int64, C.c_int64, _f64p,
                                    C.c_double, C.c_double, C.c_int64, C.c_int64,
                                    _f64p]
        L.orc_ring.argtypes = [_f32p, C.c_int64, C.c_int64, C.c_int64]
        L.orc_bp_compat_geom.argtypes = [_f32p, C.c_int64, C.c_int64, _f32p, C.c_float,
                                         C.c_float, C.c_int64, C.c_int64, C.c_float, C.c_float,
                                         C.c_float, _f32p]
        L.orc_bp_linear_geom.argtypes = [_f64p, C.c_int64, C.c_int64, _f64p, C.c_double,
                                         C.c_double, C.c_int64, C.c_int64, C.c_float, C.c_float,
                                         C.c_float, _f64p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(
                "oracle/_ref/libctcl_ref.so was not built (reference sources absent)")
        R = C.CDLL(REF_PATH)
        R.ref_ctcl_fbp.restype = C.c_int
        R.ref_ctcl_fbp.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p,
                                   C.c_float, C.c_float, C.c_int64, C.c_int64,
                                   C.c_int]
        R.ref_ctcl_fbp_rows.restype = C.c_int
        R.ref_ctcl_fbp_rows.argtypes = [_f32p, _f32p, C.c_int, C.c_int, _f32p,
                                        C.c_float, C.c_float,
                                        np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS"),
                                        C.c_int64, C.c_int]
        _ref = R
    return _ref


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------- set-up
def padded_width(W: int) -> int:
    return int(lib().orc_padded_width(W))


def filter_window(ftype: int, param: float, P: int, W: int,
                  contrast: int = PHS, fp64: bool = False) -> np.ndarray:
    out = np.zeros(P, np.float64 if fp64 else np.float32)
    rc = lib().orc_filter_fill(ftype, param, P, W, contrast,
                               None if fp64 else _ptr(out),
                               _ptr(out) if fp64 else None)
    if rc:
        raise ValueError("bad filter")
    return out


def arc(anarc: float, N: int) -> float:
    return float(lib().orc_arc(anarc, N))


def angle_table(anarc: float, N: int) -> np.ndarray:
    tab = np.zeros(2 * N, np.float32)
    lib().orc_angle_table(anarc, N, tab)
    return tab


def angle_table_list(angles) -> np.ndarray:
    th = np.ascontiguousarray(angles, np.float64)
    tab = np.zeros(2 * th.size, np.float32)
    lib().orc_angle_table_list(th, th.size, tab)
    return tab


def angle_table_f64(anarc: float, N: int) -> np.ndarray:
    tab = np.zeros(2 * N, np.float64)
    lib().orc_angle_table_f64(anarc, N, tab)
    return tab


def rec_cof(pixel_size: float = 0.0, lam: float = 0.0) -> float:
    return float(lib().orc_rec_cof(pixel_size, lam))


def in_mask(j: int, i: int, W: int, center: float) -> bool:
    return bool(lib().orc_in_mask(j, i, W, center))


def mask(W: int, center: float) -> np.ndarray:
    """Pixel mask of the reference (lct.cpp:693-707), vectorised in float32."""
    hp = W // 2
    c = np.float32(center)
    ac = np.float32(abs(c))
    i = np.arange(W)
    j = np.arange(W)[:, None]
    ip2 = ((i - hp) ** 2).astype(np.float32)
    col_ok = ~((i.astype(np.float32) <= ac) |
               (i.astype(np.float32) >= (np.float32(W) - ac) - np.float32(1)))
    ijp2 = (j - hp).astype(np.float32) - c
    ijp2 = ijp2 * ijp2
    ijp2 = ijp2 + ip2
    hpc = np.float32(hp) + c
    hmc = np.float32(hp) - c
    jf = j.astype(np.float32)
    out = ((jf <= hpc) & (ijp2 >= hpc * hpc)) | ((jf >= hpc) & (ijp2 >= hmc * hmc))
    return col_ok & ~out


# --------------------------------------------------------------- ring filter
def ring(x: np.ndarray, box: int) -> np.ndarray:
    """RingFilter::apply (lct.cpp:295-327), no mask; returns a corrected copy."""
    y = np.ascontiguousarray(x, np.float32).copy()
    lib().orc_ring(y, y.shape[0], y.shape[1], box)
    return y


# --------------------------------------------------------------- filter
def deabs(x: np.ndarray) -> np.ndarray:
    y = np.ascontiguousarray(x, np.float32).copy()
    if lib().orc_deabs(y, y.size):
        raise ValueError("Bad absorption data (maximum is sub-zero).")
    return y


def prepare_sino(x: np.ndarray, P: int, contrast: int, G: np.ndarray,
                 fp64: bool = False):
    """prepare_sino (lct.cpp:569-597).  Returns the filtered N*W sinogram
    (float32 in compat form, float64 in the fp64 form).  ``x`` is not
    modified."""
    x = np.ascontiguousarray(x, np.float32).copy()
    N, W = x.shape
    q = np.zeros((N, W), np.float64 if fp64 else np.float32)
    Gc = np.ascontiguousarray(G, np.float64 if fp64 else np.float32)
    rc = lib().orc_prepare_sino(x, N, W, P, contrast,
                                None if fp64 else _ptr(Gc),
                                _ptr(Gc) if fp64 else None,
                                None if fp64 else _ptr(q),
                                _ptr(q) if fp64 else None)
    if rc:
        raise ValueError("Bad absorption data (maximum is sub-zero).")
    return q


# --------------------------------------------------------------- backprojection
def bp_compat(q: np.ndarray, tab: np.ndarray, center: float, rec_cof: float = 1.0,
              rows: tuple[int, int] | None = None) -> np.ndarray:
    """reconstructOnCPU (lct.cpp:688-729).  float32 ``q`` -> float32 slice with
    float accumulation; float64 ``q`` -> float64 slice with double accumulation
    (indices still from the reference's float expression)."""
    N, W = q.shape
    r0, r1 = rows if rows else (0, W)
    tab = np.ascontiguousarray(tab, np.float32)
    if q.dtype == np.float64:
        qd = np.ascontiguousarray(q)
        out = np.zeros((r1 - r0, W), np.float64)
        lib().orc_bp_compat(None, _ptr(qd), N, W, tab, center, rec_cof, r0, r1,
                            None, _ptr(out))
    else:
        qf = np.ascontiguousarray(q, np.float32)
        out = np.zeros((r1 - r0, W), np.float32)
        lib().orc_bp_compat(_ptr(qf), None, N, W, tab, center, rec_cof, r0, r1,
                            _ptr(out), None)
    return out


def bp_linear(qd: np.ndarray, tab64: np.ndarray, center: float,
              rec_cof: float = 1.0, rows: tuple[int, int] | None = None) -> np.ndarray:
    N, W = qd.shape
    r0, r1 = rows if rows else (0, W)
    out = np.zeros((r1 - r0, W), np.float64)
    lib().orc_bp_linear(np.ascontiguousarray(qd, np.float64), N, W,
                        np.ascontiguousarray(tab64, np.float64), center, rec_cof,
                        r0, r1, out)
    return out


def geometry(W: int, rows: int, cols: int, pixel: float = 1.0, shift_row: float = 0.0,
             shift_col: float = 0.0):
    """(oj, oi, p) of an output grid of rows x cols pixels of pitch `pixel`
    (detector pixels), centred like the reference's W x W grid and shifted by
    (shift_row, shift_col) output pixels; float32 values."""
    p = np.float32(pixel)
    oj = np.float32((W - 1) / 2.0 - float(p) * ((rows - 1) / 2.0 - shift_row))
    oi = np.float32((W - 1) / 2.0 - float(p) * ((cols - 1) / 2.0 - shift_col))
    return float(oj), float(oi), float(p)


def bp_compat_geom(q: np.ndarray, tab: np.ndarray, center: float, rec_cof: float, rows: int,
                   cols: int, oj: float, oi: float, p: float) -> np.ndarray:
    N, W = q.shape
    out = np.zeros((rows, cols), np.float32)
    lib().orc_bp_compat_geom(np.ascontiguousarray(q, np.float32), N, W,
                             np.ascontiguousarray(tab, np.float32), center, rec_cof, rows, cols,
                             oj, oi, p, out)
    return out


def bp_linear_geom(qd: np.ndarray, tab64: np.ndarray, center: float, rec_cof: float, rows: int,
                   cols: int, oj: float, oi: float, p: float) -> np.ndarray:
    N, W = qd.shape
    out = np.zeros((rows, cols), np.float64)
    lib().orc_bp_linear_geom(np.ascontiguousarray(qd, np.float64), N, W,
                             np.ascontiguousarray(tab64, np.float64), center, rec_cof, rows, cols,
                             oj, oi, p, out)
    return out


def ref_fbp(q: np.ndarray, tab: np.ndarray, center: float, coeff: float = 1.0,
            rows: tuple[int, int] | None = None, nthreads: int = 1) -> np.ndarray:
    """The reference's ct.cl kernel run on the host over rows [r0, r1)."""
    N, W = q.shape
    r0, r1 = rows if rows else (0, W)
    slice_ = np.zeros((W, W), np.float32)
    ref_lib().ref_ctcl_fbp(np.ascontiguousarray(q, np.float32), slice_, W, N,
                           np.ascontiguousarray(tab, np.float32), center, coeff,
                           r0, r1, nthreads)
    return slice_[r0:r1]


def ref_fbp_rows(q: np.ndarray, tab: np.ndarray, center: float, coeff: float,
                 rows, out: np.ndarray, nthreads: int = 1) -> np.ndarray:
    """The reference's ct.cl kernel on the listed rows, written into the full
    W x W array `out` (reused across calls)."""
    N, W = q.shape
    rows = np.ascontiguousarray(rows, np.int64)
    assert out.shape == (W, W) and out.dtype == np.float32 and rows.min() >= 0 and rows.max() < W
    ref_lib().ref_ctcl_fbp_rows(np.ascontiguousarray(q, np.float32), out, W, N,
                                np.ascontiguousarray(tab, np.float32), center, coeff, rows,
                                rows.size, nthreads)
    return out


# --------------------------------------------------------------- full path
def reconstruct(sino: np.ndarray, contrast: int = PHS, ftype: int = 1,
                fparam: float = 0.0, arc_deg: float = 180.0, center: float = 0.0,
                pixel_size: float = 0.0, lam: float = 0.0, P: int | None = None,
                fp64: bool = False) -> np.ndarray:
    """CTrec::reconstruct (lct.cpp:649-685) on the CPU path."""
    N, W = sino.shape
    P = P or padded_width(W)
    G = filter_window(ftype, fparam, P, W, contrast, fp64=fp64)
    q = prepare_sino(sino, P, contrast, G, fp64=fp64)
    tab = angle_table(arc_deg, N)
    return bp_compat(q, tab, center, rec_cof(pixel_size, lam))
