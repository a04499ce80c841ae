"""CPU oracle for the ctas FBP hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference
legs of bench.py may import this package.  It wraps two host libraries built by
``oracle/Makefile``:

* ``_build/liboracle.so`` -- fbp_oracle.c, the C restatement of the reference
  algorithm (ctas src/common/lct.cpp:122-209, 280-291, 470-517, 558-597,
  688-729 and src/common/physical.world.cpp:88-100) in FP32-compatible and
  FP64 forms, and of the rotation-axis metrics (lct.cpp:863-913, 1246-1252);
* ``_ref/libctcl_ref.so`` -- the reference's own backprojection kernel
  (ctas src/common/ct.cl:5-44) compiled for the host;
* ``_ref/liblct_shipped.so`` and ``_ref/liblct_o2.so`` -- the reference's
  reconstruction code itself (src/common/lct.cpp with the library files it
  needs) compiled in place, as shipped (-ffast-math, no -O) and at -O2, over
  the stand-in headers of ``shim/`` (no OpenCL device, FFTW in double), with
  ``ref_lct_driver.cpp`` giving C entry points to ``CTrec``, ``RingFilter``,
  ``ts_add`` and ``raxis``.

The ``_ref`` libraries exist only where the reference sources were present
when the oracle was built (``make ref lct REFERENCE_ROOT=...``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libctcl_ref.so")
LCT_PATHS = {"shipped": os.path.join(HERE, "_ref", "liblct_shipped.so"),
             "o2": os.path.join(HERE, "_ref", "liblct_o2.so")}
# the reference's limit<T> extracted from external.world.cpp (oracle/Makefile)
LIMIT_PATH = os.path.join(HERE, "_ref", "liblimit_ref.so")

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
_lct = {}


def build(reference_root: str | None = None) -> None:
    """Build the oracle; with ``reference_root`` (a ctas source tree, default
    the environment variable CTAS_REFERENCE_ROOT) also the ``_ref`` libraries
    compiled from the reference's own sources."""
    root = reference_root or os.environ.get("CTAS_REFERENCE_ROOT")
    targets = ["all"]
    extra = []
    if root and os.path.exists(os.path.join(root, "src", "common", "lct.cpp")):
        targets += ["ref", "lct"]
        if os.path.exists(os.path.join(os.path.dirname(HERE), "ctas_b200", "libctas_fbp.so")):
            targets.append("shim-blitz")
        extra.append(f"REFERENCE_ROOT={os.path.abspath(root)}")
    subprocess.run(["make", "-s", "-C", HERE, *targets, *extra], check=True)
    if extra:
        # optional: limit<T> is extracted from a file the other targets do not
        # read; without it the tests that use it skip
        subprocess.run(["make", "-s", "-C", HERE, "limit", *extra], check=False)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
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
        L.orc_set_index_rule.argtypes = [C.c_int]
        L.orc_index_rule.restype = C.c_int
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
        L.orc_ag_metric.restype = C.c_float
        L.orc_ag_metric.argtypes = [_f32p, C.c_int64, C.c_float, C.c_float,
                                    C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.orc_filter_fill_plain.restype = C.c_int
        L.orc_filter_fill_plain.argtypes = [C.c_int, C.c_float, C.c_int64, _f32p]
        L.orc_ts_add.argtypes = [_f32p, _f32p, C.c_int64, C.c_int64, _f32p, C.c_float,
                                 C.c_int, C.c_float, C.c_int]
        L.orc_limit.restype = C.c_int
        L.orc_limit.argtypes = [_f32p, C.c_int64, C.c_int, C.c_float, C.c_float, C.c_void_p]
        L.orc_pair_sq.restype = C.c_double
        L.orc_pair_sq.argtypes = [_f32p, _f32p, C.c_int64, C.c_int64, C.c_float, C.c_int64]
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
# Rounding order of the index expression's first term (fbp_oracle.c,
# orc_set_index_rule): "ctcl" = ct.cl:36-37 as written, c + ((1-s)-co)*hp;
# "shipped" = lct.cpp:711-712 as the reference's -ffast-math build compiles it,
# c + (1-(s+co))*hp.
INDEX_RULES = {"ctcl": 0, "shipped": 1}


def _set_rule(rule: str) -> None:
    lib().orc_set_index_rule(INDEX_RULES[rule])


def bp_compat(q: np.ndarray, tab: np.ndarray, center: float, rec_cof: float = 1.0,
              rows: tuple[int, int] | None = None, rule: str = "ctcl") -> np.ndarray:
    """reconstructOnCPU (lct.cpp:688-729).  float32 ``q`` -> float32 slice with
    float accumulation; float64 ``q`` -> float64 slice with double accumulation
    (indices still from the reference's float expression, in the rounding
    order ``rule``)."""
    N, W = q.shape
    r0, r1 = rows if rows else (0, W)
    tab = np.ascontiguousarray(tab, np.float32)
    _set_rule(rule)
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
                   cols: int, oj: float, oi: float, p: float, rule: str = "ctcl") -> np.ndarray:
    N, W = q.shape
    out = np.zeros((rows, cols), np.float32)
    _set_rule(rule)
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
                fp64: bool = False, rule: str = "ctcl") -> np.ndarray:
    """CTrec::reconstruct (lct.cpp:649-685) on the CPU path."""
    N, W = sino.shape
    P = P or padded_width(W)
    G = filter_window(ftype, fparam, P, W, contrast, fp64=fp64)
    q = prepare_sino(sino, P, contrast, G, fp64=fp64)
    tab = angle_table(arc_deg, N)
    return bp_compat(q, tab, center, rec_cof(pixel_size, lam), rule=rule)


# --------------------------------------------------------------- axis search
# Restatement of the rotation-axis search (ctas src/common/lct.cpp:792-1297)
# with the reference's float / double conversions written out.  The
# per-trial metrics come from fbp_oracle.c; the control flow is here.
f32, f64 = np.float32, np.float64


def step_rad(anarc: float, N: int) -> np.float32:
    """angO (lct.cpp:478-484)."""
    r = f32(anarc)
    if r > 1.0 and N > 1:
        r = f32(r / f32(N - 1))
    return f32(f64(r) * (np.pi / 180))


def ag_sigma(anarc: float, N: int, W: int) -> np.float32:
    """sigma = angO(anarc, N) * W / M_PI (lct.cpp:836)."""
    return f32(f64(f32(step_rad(anarc, N) * f32(W))) / np.pi)


def ag_metric(slice_: np.ndarray, centre: float, sigma: float):
    """AverageGradient::apply after the reconstruction: (value, double sum, count)."""
    sl = np.ascontiguousarray(slice_, np.float32)
    W = sl.shape[0]
    s = C.c_double()
    n = C.c_int64()
    v = lib().orc_ag_metric(sl, W, f32(centre), f32(sigma), C.byref(s), C.byref(n))
    return f32(v), s.value, n.value


class AgOracle:
    """AverageGradient (lct.cpp:800-915) on the CPU path: ABS contrast, RAMP
    window, the reference's padding rule and angle table."""

    def __init__(self, sino: np.ndarray, anarc: float = 180.0, rule: str = "ctcl"):
        sino = np.ascontiguousarray(sino, np.float32)
        self.rule = rule
        self.N, self.W = sino.shape
        P = padded_width(self.W)
        G = filter_window(FILTERS["RAMP"], 0.0, P, self.W, ABS)
        self.q = prepare_sino(sino, P, ABS, G)
        self.tab = angle_table(anarc, self.N)
        self.sigma = ag_sigma(anarc, self.N, self.W)
        self.calls = 0

    def centre(self, axis_r: float) -> np.float32:
        # const float centre = axisR - 0.5*(ish(1)-1);
        return f32(f64(f32(axis_r)) - 0.5 * (self.W - 1))

    def slice(self, axis_r: float) -> np.ndarray:
        c = self.centre(axis_r)
        if abs(c) >= self.W // 2:
            raise ValueError("centre out of range")
        return bp_compat(self.q, self.tab, float(c), 1.0, rule=self.rule)

    def apply(self, axis_r: float) -> np.float32:
        self.calls += 1
        c = self.centre(axis_r)
        return ag_metric(self.slice(axis_r), c, self.sigma)[0]


def improve_me(eps, vaxS, errS, idx, cdir, getvx):
    """improveMe (lct.cpp:1114-1134)."""
    eps = f32(eps)
    ab = [f32(vaxS[idx - cdir]), f32(vaxS[idx + cdir])]  # aa, bb
    rf = f32(vaxS[idx])
    vl = f32(errS[idx])
    while abs(f32(ab[0] - rf)) > eps or abs(f32(rf - ab[1])) > eps:
        afar = abs(f32(ab[0] - rf)) > abs(f32(rf - ab[1]))
        lo, hi = (0, 1) if afar else (1, 0)
        x = f32(f32(rf + ab[lo]) / f32(2))
        vx = f32(getvx(x))
        if vl <= vx:
            ab[lo] = x
        else:
            vl = vx
            ab[hi] = rf
            rf = x
    return rf


def raxis_pair(p0: np.ndarray, p180: np.ndarray, max_dev: float) -> np.float32:
    """raxis(proj0, proj180, maxDev) (lct.cpp:1217-1297)."""
    p0 = np.ascontiguousarray(p0, np.float32)
    p180 = np.ascontiguousarray(p180, np.float32)
    max_dev = f32(max_dev)
    if max_dev < 0 or max_dev > 0.5:
        raise ValueError("Invalid maximum relative shift")
    rows, W = p0.shape
    cent = f32(0.5 * (W - 1))
    proj = np.zeros(W, np.float32)
    for j in range(rows):
        t = np.abs(p0[j].astype(np.float64) - 1.0) + np.abs(p180[j].astype(np.float64) - 1.0)
        proj = (proj.astype(np.float64) + t).astype(np.float32)
    s = 0.0
    si = 0.0
    for i in range(W):
        s += float(proj[i])
        si += float(f32(f32(i) * proj[i]))
    ssum = f32(s)
    if ssum == 0:
        raise ValueError("Impossible input projection averaging to zero.")
    fcr = f32(si / f64(ssum))
    stpsz = 16
    stf = f32(1.0) if max_dev == 0 else f32(f32(max_dev * f32(W)) / f32(stpsz))
    steps = int(f32(f32(1) + f32(f32(2) * stf)))
    if steps < 3:
        raise ValueError("fewer than 3 trials")
    a0 = sum(float(v) for v in p180[:, W - 1])
    a1 = sum(float(v) for v in p180[:, 0])
    aver = f32((a0 + a1) / (2 * rows))

    def calc(x):
        xs = int(np.trunc(f64(x)))
        if abs(xs) >= W:
            raise ValueError("trial shift of a whole width")
        return f32(np.sqrt(lib().orc_pair_sq(p0, p180, rows, W, aver, xs)))

    vaxS = [f32(f32(f32(2) * f32(fcr - cent)) + f32(stpsz * (ii - (steps - 1) // 2)))
            for ii in range(steps)]
    errS = [calc(v) for v in vaxS]
    idx = 0
    minval = f32(np.finfo(np.float32).max)
    for i in range(1, steps - 1):
        if errS[i] < errS[i - 1] and errS[i] < errS[i + 1] and errS[i] < minval:
            idx = i
            minval = errS[i]
    if minval != f32(np.finfo(np.float32).max):
        return f32(f64(cent) + 0.5 * f64(improve_me(1.0, vaxS, errS, idx, 1, calc)))
    idx = 0 if errS[0] < errS[steps - 1] else steps - 1
    cdir = -1 if idx == 0 else 1
    minval = errS[idx]
    maxSteps = int(f32(f32(f32(W // 2) - f32(f32(cdir) * vaxS[idx])) / f32(stpsz)))
    if maxSteps <= 0:
        raise ValueError("Failed to calculate rotation centre.")
    vaxS2 = [vaxS[idx - cdir], vaxS[idx]] + [f32(0)] * maxSteps
    errS2 = [errS[idx - cdir], errS[idx]] + [f32(0)] * maxSteps
    idx2 = 1
    for i in range(maxSteps):
        vaxS2[i + 2] = f32(vaxS[idx] + f32(cdir * (i + 1) * stpsz))
        errS2[i + 2] = calc(vaxS2[i + 2])
        if errS2[i + 2] < minval:
            minval = errS2[i + 2]
            idx2 = i + 2
        else:
            break
    if idx2 == maxSteps + 1:
        raise ValueError("Failed to calculate rotation centre.")
    return f32(f64(cent) + 0.5 * f64(improve_me(1.0, vaxS2, errS2, idx2, cdir, calc)))


def raxis(sino: np.ndarray, anarc: float, max_dev: float, algo: int = 0):
    """raxis(Map &sino, anarc, maxDev, algo) (lct.cpp:1137-1212).  Returns
    (axis, number of average-gradient evaluations).  The march after the grid
    runs in order (the reference's threads may reorder it)."""
    sino = np.ascontiguousarray(sino, np.float32)
    N, W = sino.shape
    if N < 3 or W < 3:
        raise ValueError("Shape of input sinogram is less than minimal")
    a = arc(anarc, N)
    if a == 0:
        raise ValueError("Zero sinogram arc.")
    if abs(a) < np.pi:
        raise ValueError("Sinogram arc is less than 180 degree.")
    max_dev = f32(max_dev)
    if max_dev < 0 or max_dev > f32(0.25):
        raise ValueError("Invalid maximum relative shift")
    cent = f32(0.5 * (W - 1))

    def raxisQ():
        idx180 = int(f64(N - 1) * np.pi / f64(abs(f32(arc(anarc, N)))))
        nofln = N - idx180
        row0 = (sino[:nofln] + f32(1)).astype(np.float32)
        row180 = (sino[idx180:idx180 + nofln] + f32(1)).astype(np.float32)
        return raxis_pair(row0, row180, min(max_dev, f32(0.5)))

    if algo == 0:
        return raxisQ(), 0
    if algo == 1:
        fcr = cent
    elif algo == 2:
        fcr = raxisQ()
    elif algo == 3:
        pl = np.zeros(W, np.float32)
        for j in range(N):
            pl = (pl + sino[j]).astype(np.float32)
        threshold = f32(0.1 * f64(pl.max()) + 0.9 * f64(pl.min()))
        above = np.nonzero(pl > threshold)[0]
        if above.size == 0:
            raise ValueError("constant projection profile")
        fcr = f32(f32(f32(above[0]) + f32(above[-1])) / f32(2))
    else:
        raise ValueError("Unknown algorithm")
    if f32(abs(f32(fcr - cent)) / f32(W)) > max_dev:
        raise ValueError("Rotation axis relative shift is larger than maximum shift")
    rbxsz = f32(1.0 - 2.0 * f64(f32(max_dev + f32(abs(f32(fcr - cent)) / f32(W)))))
    if rbxsz < 0.5:
        raise ValueError("Relative box size is less than miminum window of 0.5")
    stpsz = 8
    stf = f32(1.0) if max_dev == 0 else f32(f32(max_dev * f32(W)) / f32(stpsz))
    steps = int(f32(f32(1) + f32(f32(2) * stf)))
    if steps < 3:
        raise ValueError("fewer than 3 trials")
    ag = AgOracle(sino, anarc)
    coffee = f32(fcr - cent)
    hf = (steps - 1) // 2
    vaxS = [f32(coffee + f32(stpsz * (i - hf))) for i in range(steps)]
    errS = [ag.apply(f32(cent + v)) for v in vaxS]
    idxM = 0
    minval = f32(np.finfo(np.float32).max)
    for i in range(1, steps - 1):
        c = errS[i]
        if c < errS[i - 1] and c < errS[i + 1] and c < minval:
            idxM = i
            minval = c
    cdir = 1
    if not idxM:
        idx = 0 if errS[0] < errS[steps - 1] else steps - 1
        cdir = -1 if idx == 0 else 1
        coffee2 = int(vaxS[idx - cdir * 2])
        q = abs(cdir * coffee2) // stpsz * (1 if cdir * coffee2 >= 0 else -1)  # C division
        maxSteps = int(f32(f32(f32(W) * f32(0.25)) - f32(q)))
        if maxSteps <= 0:
            raise ValueError("Impossible number of steps.")
        v2 = [f32(0)] * maxSteps
        e2 = [f32(0)] * maxSteps
        for i in range(maxSteps):
            v2[i] = f32(f32(coffee2) + f32(stpsz * i * cdir))
            e2[i] = ag.apply(f32(cent + v2[i]))
            if e2[i] < minval:
                minval = e2[i]
                idxM = i
            else:
                break
        if idxM == maxSteps - 1 or idxM == 0:
            return fcr, ag.calls
        vaxS, errS = v2, e2
    rf = improve_me(0.25, vaxS, errS, idxM, cdir, lambda x: ag.apply(f32(cent + x)))
    return f32(cent + rf), ag.calls


# --------------------------------------------------------------- tomosynthesis
def filter_fill_plain(ftype: int, param: float, n: int) -> np.ndarray:
    """Filter::fill(filt, n) (lct.cpp:122-209) for any length n."""
    out = np.zeros(n, np.float32)
    if lib().orc_filter_fill_plain(ftype, param, n, out):
        raise ValueError("bad filter length")
    return out


def ts_add(proj: np.ndarray, result: np.ndarray, ftype: int, fparam: float, center: float,
           contrast: int, angle: float, plane: int):
    """ts_add (lct.cpp:731-787) with an exact (FP64) row filter.  Returns the
    projection as the reference leaves it and the accumulated result (new
    arrays; the inputs are not modified)."""
    p = np.ascontiguousarray(proj, np.float32).copy()
    r = np.ascontiguousarray(result, np.float32).copy()
    rows, n = p.shape
    fw = filter_fill_plain(ftype, fparam, n)
    lib().orc_ts_add(p, r, rows, n, fw, f32(center), contrast, f32(angle), int(plane))
    return p, r


# --------------------------------------------------------------- volume writer
SAMPLE_TYPES = {8: np.uint8, -8: np.int8, 16: np.uint16, -16: np.int16, 32: np.uint32,
                -32: np.int32, 64: np.uint64, -64: np.int64}


def limit(image: np.ndarray, bpp: int, mincon: float = 0.0, maxcon: float = 0.0) -> np.ndarray:
    """limit<T> (external.world.cpp:69-90): one image -> integer samples of
    bpp bits (negative = signed); mincon == maxcon uses the image's range."""
    img = np.ascontiguousarray(image, np.float32)
    out = np.zeros(img.shape, SAMPLE_TYPES[bpp])
    if lib().orc_limit(img.reshape(-1), img.size, bpp, f32(mincon), f32(maxcon),
                       out.ctypes.data_as(C.c_void_p)):
        raise ValueError("bad bits per sample")
    return out


def ref_limit_available() -> bool:
    return os.path.exists(LIMIT_PATH)


def ref_limit(image: np.ndarray, bpp: int, mincon: float = 0.0, maxcon: float = 0.0) -> np.ndarray:
    """The reference's own limit<T> (external.world.cpp:69-90, built from the
    file where it lies, reference flags) for bpp 8, -8, 16, -16."""
    img = np.ascontiguousarray(image, np.float32)
    if img.ndim != 2:
        raise ValueError("one 2-D image")
    L = C.CDLL(LIMIT_PATH)
    L.ref_limit.restype = C.c_int
    L.ref_limit.argtypes = [_f32p, C.c_long, C.c_long, C.c_int, C.c_float, C.c_float, C.c_void_p]
    out = np.zeros(img.shape, SAMPLE_TYPES[bpp])
    if L.ref_limit(img.reshape(-1), img.shape[0], img.shape[1], bpp, f32(mincon), f32(maxcon),
                   out.ctypes.data_as(C.c_void_p)):
        raise ValueError("bad bits per sample")
    return out


# ------------------------------------------- the reference's own CTrec (oracle/_ref)
def lct_available(variant: str = "shipped") -> bool:
    return os.path.exists(LCT_PATHS[variant])


def lct_lib(variant: str = "shipped"):
    """The reference's lct.cpp built in place (``shipped``: its own flags,
    -ffast-math with no -O; ``o2``: -O2 -ffast-math), through ref_lct_driver.cpp."""
    if variant not in _lct:
        path = LCT_PATHS[variant]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} was not built (reference sources absent)")
        L = C.CDLL(path)
        f, i, lg, fp = C.c_float, C.c_int, C.c_long, _f32p
        L.ref_lct_last_error.restype = C.c_char_p
        L.ref_lct_filter_fill.argtypes = [i, i, f, fp]
        L.ref_lct_reconstruct.argtypes = [fp, fp, lg, lg, i, i, f, f, f, f, f]
        L.ref_lct_sino_repeat.argtypes = [fp, fp, lg, lg, i, i, f, f, _f32p, i, f, f]
        L.ref_lct_ring.argtypes = [fp, lg, lg, lg]
        L.ref_lct_ts_add.argtypes = [fp, fp, lg, lg, i, f, f, i, f, i]
        L.ref_lct_raxis.argtypes = [fp, lg, lg, f, f, i, C.POINTER(C.c_float)]
        L.ref_lct_ag_metric.argtypes = [fp, lg, lg, f, _f32p, i, _f32p]
        L.ref_lct_mmap_threshold.argtypes = [i]
        L.ref_lct_reconstruct_stack.argtypes = [fp, C.c_void_p, lg, lg, lg, i, i, f, f, f, f,
                                                f, i, C.POINTER(C.c_double)]
        _lct[variant] = L
    return _lct[variant]


def _lct_check(L, rc):
    if rc != 0:
        raise RuntimeError(f"reference code failed ({rc}): {L.ref_lct_last_error().decode()}")


def _trailing(sino: np.ndarray) -> np.ndarray:
    """n*w + 1 floats, the last one 0: the reference's padding reads one float
    past the last row (lct.cpp:579-584)."""
    N, W = sino.shape
    buf = np.zeros(N * W + 1, np.float32)
    buf[:N * W] = np.asarray(sino, np.float32).ravel()
    return buf


def lct_filter_fill(ftype: int, param: float, P: int, variant: str = "shipped") -> np.ndarray:
    """Filter::fill(window, P) (lct.cpp:122-209), before the P/W scaling."""
    L = lct_lib(variant)
    out = np.zeros(P, np.float32)
    _lct_check(L, L.ref_lct_filter_fill(P, ftype, param, out))
    return out


def lct_reconstruct(sino: np.ndarray, contrast: int = PHS, ftype: int = 1, fparam: float = 0.0,
                    arc: float = 180.0, center: float = 0.0, pixel_size: float = 0.0,
                    lam: float = 0.0, variant: str = "shipped"):
    """CTrec(shape, contrast, arc, Filter(ftype, fparam)).setPhysics(...) then
    reconstruct(sino, slice, center) (lct.cpp:487-526, 558-566, 649-685, 688-729).
    Returns (filtered sinogram as the reference leaves it in place, slice)."""
    L = lct_lib(variant)
    N, W = sino.shape
    buf = _trailing(sino)
    out = np.zeros((W, W), np.float32)
    _lct_check(L, L.ref_lct_reconstruct(buf, out, N, W, contrast, ftype, fparam, arc, center,
                                        pixel_size, lam))
    return buf[:N * W].reshape(N, W), out


def lct_sino_repeat(sino: np.ndarray, centers, contrast: int = PHS, ftype: int = 1,
                    fparam: float = 0.0, arc: float = 180.0, pixel_size: float = 0.0,
                    lam: float = 0.0, variant: str = "shipped"):
    """CTrec::sino then repeat(slice, c) per centre (lct.cpp:600-647)."""
    L = lct_lib(variant)
    N, W = sino.shape
    cs = np.ascontiguousarray(centers, np.float32)
    buf = _trailing(sino)
    out = np.zeros((len(cs), W, W), np.float32)
    _lct_check(L, L.ref_lct_sino_repeat(buf, out, N, W, contrast, ftype, fparam, arc, cs, len(cs),
                                        pixel_size, lam))
    return buf[:N * W].reshape(N, W), out


def lct_ring(sino: np.ndarray, box: int, variant: str = "shipped") -> np.ndarray:
    """RingFilter(W, box).apply(sino) (lct.cpp:295-327)."""
    L = lct_lib(variant)
    x = np.ascontiguousarray(sino, np.float32).copy()
    _lct_check(L, L.ref_lct_ring(x, x.shape[0], x.shape[1], box))
    return x


def lct_ts_add(proj: np.ndarray, result: np.ndarray, ftype: int, fparam: float, center: float,
               contrast: int, angle: float, plane: int, variant: str = "shipped"):
    """ts_add (lct.cpp:739-787).  Returns (filtered projection, result + its
    backprojection)."""
    L = lct_lib(variant)
    p = np.ascontiguousarray(proj, np.float32).copy()
    r = np.ascontiguousarray(result, np.float32).copy()
    _lct_check(L, L.ref_lct_ts_add(p, r, p.shape[0], p.shape[1], ftype, fparam, center,
                                   contrast, angle, plane))
    return p, r


def lct_ag_metric(sino: np.ndarray, arc: float, axes, variant: str = "shipped") -> np.ndarray:
    """AverageGradient(sino, arc).apply(axis) (lct.cpp:804-915) per axis
    position (detector coordinate of the rotation axis).  The reference reads
    one float past a sinogram copy it allocates itself; call
    ``lct_lib().ref_lct_mmap_threshold(65536)`` first, in a process of its
    own, so that float is 0 (ref_lct_driver.cpp explains)."""
    L = lct_lib(variant)
    s = np.ascontiguousarray(sino, np.float32)
    ax = np.ascontiguousarray(axes, np.float32)
    out = np.zeros(len(ax), np.float32)
    _lct_check(L, L.ref_lct_ag_metric(s, s.shape[0], s.shape[1], arc, ax, len(ax), out))
    return out


def lct_raxis(sino: np.ndarray, arc: float, max_dev: float, algo: int = 0,
              variant: str = "shipped") -> float:
    """raxis(sino, arc, maxDev, algo) (lct.cpp:1133-1215); only algorithm 0
    runs without OpenCL (ref_lct_driver.cpp says why)."""
    L = lct_lib(variant)
    s = np.ascontiguousarray(sino, np.float32)
    ax = C.c_float(0.0)
    _lct_check(L, L.ref_lct_raxis(s, s.shape[0], s.shape[1], arc, max_dev, algo, C.byref(ax)))
    return float(ax.value)


def lct_reconstruct_stack(sinos: np.ndarray, contrast: int, ftype: int, fparam: float, arc: float,
                          center: float, pixel_size: float = 0.0, lam: float = 0.0,
                          threads: int = 0, keep: bool = True, variant: str = "o2"):
    """The ct tool's slice loop (ct.cpp:156-236) on the reference's InThread
    pool: one CTrec clone per thread, one slice per task.  Returns (slices or
    None, wall seconds)."""
    L = lct_lib(variant)
    S, N, W = sinos.shape
    x = np.ascontiguousarray(sinos, np.float32)
    out = np.zeros((S, W, W), np.float32) if keep else None
    secs = C.c_double(0.0)
    _lct_check(L, L.ref_lct_reconstruct_stack(x, None if out is None else out.ctypes.data_as(
        C.c_void_p), S, N, W, contrast, ftype, fparam, arc, center, pixel_size, lam, threads,
        C.byref(secs)))
    return out, float(secs.value)
