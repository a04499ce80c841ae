"""CPU-side checks of the C ABI: the library loads, exports every declared
symbol, and its host-side set-up (padding rule, filter names and windows,
angle table, physics coefficient) agrees with the oracle.  No GPU needed."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from ctas_b200 import _lib, ct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = "".join(open(p).read() for p in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctas_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    L = _lib.load()
    for s in syms:
        assert hasattr(L, s)
    assert set(syms) == set(_lib.SIGNATURES)


@pytest.mark.parametrize("prog", ["shim_usage.cpp", "axis_usage.cpp", "ts_usage.cpp",
                                  "volume_usage.cpp"])
def test_cpp_shim_compiles(prog):
    src = os.path.join(ROOT, "tests", "cpp", prog)
    res = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                          src], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_tile_count():
    from test_gpu_parity import N_TILES
    assert ct.tile_count() == N_TILES


def test_padded_width_matches_oracle():
    for w in (2, 3, 7, 100, 512, 1024, 1536, 2048, 2560, 3072, 4096, 8192):
        assert ct.padded_width(w) == O.padded_width(w)


@pytest.mark.parametrize("name,tp", [("", 1), ("ramp", 1), ("BARLETT", 1), ("none", 0),
                                     ("Welch", 3), ("PARZEN", 4), ("hann", 5), ("HAMMING", 6),
                                     ("blackman", 7), ("LANCKZOS", 8), ("kaiser", 9),
                                     ("gauss", 10), ("shepp-logan", 100), ("cosine", 101)])
def test_filter_names(name, tp):
    v = C.c_int32()
    assert _lib.load().ctas_filter_from_name(name.encode(), C.byref(v)) == 0
    assert v.value == tp


def test_filter_errors():
    with pytest.raises(ct.CtasError) as e:
        ct.Filter("nosuch")
    assert e.value.code == _lib.E_FILTER and "does not describe any known filter" in e.value.msg
    with pytest.raises(ct.CtasError):
        ct.Filter("KAISER", -1.0)
    with pytest.raises(ct.CtasError):
        ct.Filter("GAUSS", 0.0)
    f = ct.Filter.parse("GAUSS:0.5")
    assert f.filter() == 10 and abs(f.param() - 0.5) < 1e-7
    assert ct.Filter.parse("hann").name() == "HANN"
    with pytest.raises(ct.CtasError):
        ct.Filter.parse("hann:abc")


def test_contrast_names():
    for s, v in (("A", 0), ("abs", 0), ("REFRACTION", 1), ("p", 2), ("phase", 2), ("FLT", 3)):
        assert ct.Contrast(s).contrast() == v
    assert ct.Contrast(2).name() == "PHASE"
    with pytest.raises(ct.CtasError):
        ct.Contrast("xyz")


@pytest.mark.parametrize("ft,param", [(1, 0.0), (0, 0.0), (3, 0.0), (4, 0.0), (5, 0.0),
                                      (6, 0.0), (7, 0.0), (8, 0.0), (9, 2.0), (10, 0.7),
                                      (100, 0.0), (101, 0.0)])
@pytest.mark.parametrize("W", [64, 100, 2560])
def test_window_matches_oracle(ft, param, W):
    P = ct.padded_width(W)
    for cn in (O.PHS, O.REF):
        a = ct.window(W, cn, ft, param)
        b = O.filter_window(ft, param, P, W, cn)
        # both restate FFTW's float HC2R with an FP64 transform: agree to an ulp
        np.testing.assert_allclose(a, b, rtol=3e-7, atol=1e-7 * np.abs(b).max())
        assert np.array_equal(a[1:], a[1:][::-1])


def test_explicit_pad_window():
    a = ct.window(2560, O.PHS, 5, 0.0, pad=4096)
    b = O.filter_window(5, 0.0, 4096, 2560, O.PHS)
    np.testing.assert_allclose(a, b, rtol=3e-7, atol=1e-7 * np.abs(b).max())


@pytest.mark.parametrize("arc,N", [(180.0, 720), (180.0, 1800), (360.0, 900), (0.25, 500),
                                   (90.0, 7)])
def test_angle_table_bit_identical_to_oracle(arc, N):
    a = ct.angle_table(arc, N)
    b = O.angle_table(arc, N)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert abs(ct.arc_rad(arc, N) - O.arc(arc, N)) == 0


def test_rec_cof():
    for ps, lam in ((0.0, 0.0), (1e-6, 0.0), (0.0, 1e-10), (6.5e-6, 0.7e-10)):
        assert ct.rec_cof(ps, lam) == O.rec_cof(ps, lam)


def test_no_device_fails_loudly_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ct.CtasError) as e:
        ct.CTrec((10, 16), ct.Contrast.PHS)
    assert e.value.code == _lib.E_NODEVICE


def test_shape_errors_precede_device():
    # lct.cpp:500-503 checks come before any device work
    with pytest.raises(ct.CtasError) as e:
        ct.CTrec((10, 1), ct.Contrast.PHS)
    assert e.value.code == _lib.E_SHAPE
    with pytest.raises(ct.CtasError) as e:
        ct.CTrec((0, 16), ct.Contrast.PHS)
    assert e.value.code == _lib.E_SHAPE
