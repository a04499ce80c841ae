"""The oracle pinned to the reference's own reconstruction code.

tests/golden/lct_*.npz hold outputs of the reference's src/common/lct.cpp as
its build compiles it (-ffast-math, no -O), run through CTrec, RingFilter,
ts_add, raxis and AverageGradient (tests/golden/make_lct_golden.py; FFTW is
stood in for by a double-precision transform, oracle/shim/).  These CPU tests
check the oracle against them:

* windows (Filter::fill): bit for bit;
* filtered sinograms (prepare_sino): relative RMSE <= 1e-6 -- the FFT is the
  only difference (about one float ulp per value);
* backprojection of the reference's own filtered rows with the as-built index
  rounding ("shipped" rule): bit for bit; full path: relative RMSE <= 1e-5 and
  max |diff| <= 1e-4 of the slice's range;
* ring filter bit for bit, ts_add within 1e-6 of the range, raxis algorithm 0
  equal, the AverageGradient metric within 1e-6 relative.

Where oracle/_ref/liblct_shipped.so was built (the reference tree was
present), further tests run the reference code directly on fresh inputs.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import lct_inputs as LI  # noqa: E402
from make_lct_golden import FULL, LARGE  # noqa: E402

live = pytest.mark.skipif(not O.lct_available("shipped"),
                          reason="reference code not built here (oracle/_ref)")


def _load(name):
    return np.load(os.path.join(GOLD, f"lct_{name}.npz"))


def rel_rmse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def assert_fbp_close(got, want):
    want = np.asarray(want, np.float64)
    rng = float(want.max() - want.min()) or 1.0
    assert rel_rmse(got, want) <= 1e-5, rel_rmse(got, want)
    assert float(np.abs(np.asarray(got, np.float64) - want).max()) <= 1e-4 * rng


def large_input(name):
    N, W, cn, ft, c, photons, seed, nel, stride = LARGE[name]
    x = LI.ellipse_sino(seed, N, W, c, 180.0, n=nel, axes=(5.0, 0.23 * W),
                        rho=(0.05, 0.5) if nel == 30 else (0.1, 1.0), photons=photons)
    return x


# ------------------------------------------------------------------ fixtures
def test_windows_bitexact_vs_reference_fixture():
    d = _load("windows")
    for key in d.files:
        _, P, ft, fp = key.split("_")
        want = d[key]
        got = O.filter_fill_plain(int(ft), float(fp), int(P))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), key


def test_product_window_bitexact_vs_reference_fixture():
    """The window the device path uses (host code of the library, no GPU)."""
    from ctas_b200 import ct
    d = _load("windows")
    for key in d.files:
        _, P, ft, fp = key.split("_")
        P, ft = int(P), int(ft)
        for W in {P // 2, P // 2 - 3, P // 4 + 1} - {0, 1}:
            want = (d[key] * np.float32(np.float32(P) / np.float32(W))).astype(np.float32)
            got = ct.window(W, 2, ft, float(fp), pad=P)
            assert np.array_equal(np.asarray(got, np.float32).view(np.uint32),
                                  want.view(np.uint32)), (key, W)


@pytest.mark.parametrize("name", list(FULL))
def test_full_cases_vs_reference_fixture(name):
    d = _load(name)
    x, q_ref, sl_ref = d["sino"], d["filtered"], d["slice"]
    N, W = x.shape
    kind = FULL[name][0]
    assert np.array_equal(x, __import__("make_lct_golden").full_input(
        kind, 100 + list(FULL).index(name), N, W, float(d["center"]), float(d["arc"])))
    cn, ft, fp = int(d["contrast"]), int(d["ftype"]), float(d["fparam"])
    arc, c = float(d["arc"]), float(d["center"])
    ps, lam = float(d["pixel_size"]), float(d["lam"])
    P = O.padded_width(W)
    q = O.prepare_sino(x, P, cn, O.filter_window(ft, fp, P, W, cn))
    assert rel_rmse(q, q_ref) <= 1e-6, rel_rmse(q, q_ref)
    bp = O.bp_compat(q_ref.copy(), O.angle_table(arc, N), c, O.rec_cof(ps, lam), rule="shipped")
    assert np.array_equal(bp.view(np.uint32), sl_ref.view(np.uint32))
    assert_fbp_close(O.reconstruct(x, cn, ft, fp, arc, c, ps, lam, rule="shipped"), sl_ref)


def test_ctcl_rule_is_not_the_shipped_build():
    """ct.cl's rounding order, which the OpenCL path and a build without
    -ffast-math use, picks other samples than the reference's CPU path as
    built: the two differ well beyond the parity tolerance."""
    d = _load("c0")
    x = large_input("c0")
    N, W = x.shape
    q = O.prepare_sino(x, O.padded_width(W), O.PHS, O.filter_window(1, 0.0, O.padded_width(W), W))
    tab = O.angle_table(180.0, N)
    r = int(d["rows"][len(d["rows"]) // 2])
    a = O.bp_compat(q, tab, 0.0, 1.0, rows=(r, r + 1), rule="ctcl")
    b = O.bp_compat(q, tab, 0.0, 1.0, rows=(r, r + 1), rule="shipped")
    assert not np.array_equal(a, b)


@pytest.mark.parametrize("name", list(LARGE))
def test_large_cases_vs_reference_fixture(name):
    d = _load(name)
    x = large_input(name)
    assert LI.sha(x) == str(d["sino_sha"]), "input generator drifted"
    N, W = x.shape
    cn, ft, c = int(d["contrast"]), int(d["ftype"]), float(d["center"])
    P = O.padded_width(W)
    q = O.prepare_sino(x, P, cn, O.filter_window(ft, 0.0, P, W, cn))
    qi = d["filtered_rows_idx"]
    assert rel_rmse(q[qi], d["filtered_rows"]) <= 1e-6
    tab = O.angle_table(180.0, N)
    rows = d["rows"]
    got = np.concatenate([O.bp_compat(q, tab, c, 1.0, rows=(int(r), int(r) + 1), rule="shipped")
                          for r in rows])
    assert_fbp_close(got, d["slice_rows"])


def test_ring_bitexact_vs_reference_fixture():
    d = _load("ring")
    x = LI.normal(300, 120, 160)
    assert LI.sha(x) == str(d["sino_sha"])
    for b in (1, 3, 7):
        got = O.ring(x, b)
        assert np.array_equal(got.view(np.uint32), d[f"box{b}"].view(np.uint32)), b


def test_ts_add_vs_reference_fixture():
    d = _load("ts")
    p = d["proj"]
    res = np.zeros_like(p)
    for k, (ft, c, cn, ang, plane) in enumerate([(1, 0.0, O.PHS, 0.3, 10),
                                                 (5, 2.5, O.REF, -0.2, -5),
                                                 (6, -1.5, O.ABS, 0.1, 3)]):
        fp, res = O.ts_add(p, res, ft, 0.0, c, cn, ang, plane)
        want_f, want_r = d[f"filtered{k}"], d[f"result{k}"]
        assert np.abs(fp - want_f).max() <= 1e-6 * np.abs(want_f).max()
        assert np.abs(res - want_r).max() <= 1e-6 * (want_r.max() - want_r.min())


def test_raxis_pair_vs_reference_fixture():
    d = _load("raxis0")
    arc = 180.0 * 361 / 360
    for k, true_c in enumerate((0.0, 3.0, -5.5)):
        x = LI.ellipse_sino(310 + k, 361, 192, true_c, arc, n=8, axes=(5.0, 50.0))
        assert LI.sha(x) == str(d[f"sino_sha{k}"])
        ax, _ = O.raxis(x, arc, 0.1, 0)
        assert np.float32(ax) == d[f"axis{k}"]


def test_average_gradient_vs_reference_fixture():
    d = _load("agmetric")
    for k in range(3):
        t, arc, axes, want = d[f"trans{k}"], float(d[f"arc{k}"]), d[f"axes{k}"], d[f"metric{k}"]
        ag = O.AgOracle(t, arc, rule="shipped")
        got = np.array([ag.apply(a) for a in axes], np.float32)
        assert np.all(np.abs(got - want) <= 1e-6 * np.abs(want)), (k, got, want)


# ------------------------------------------------------- live reference code
@live
@pytest.mark.parametrize("P", [8, 64, 2048, 8192, 16384])
def test_windows_live(P):
    for ft, fp in [(0, 0.0), (1, 0.0), (3, 0.0), (4, 0.0), (5, 0.0), (6, 0.0), (7, 0.0),
                   (8, 0.0), (9, 1.5), (10, 0.7)]:
        want = O.lct_filter_fill(ft, fp, P)
        got = O.filter_fill_plain(ft, fp, P)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (P, ft)


@live
@pytest.mark.parametrize("seed,N,W,cn,ft,arc,c", [
    (1, 64, 33, O.PHS, 5, 180.0, 0.5), (2, 100, 200, O.REF, 1, 180.0, -7.25),
    (3, 77, 150, O.ABS, 6, 360.0, 4.0), (4, 120, 96, O.PHS, 7, 0.5, -2.0),
    (5, 33, 17, O.PHS, 1, 180.0, 3.0)])
def test_reconstruct_live(seed, N, W, cn, ft, arc, c):
    if cn == O.ABS:
        x = LI.transmission(seed, N, W, c)
    else:
        x = LI.ellipse_sino(seed, N, W, c, arc, n=5, axes=(2.0, W / 4.0))
    q_ref, sl_ref = O.lct_reconstruct(x, cn, ft, 0.0, arc, c)
    P = O.padded_width(W)
    q = O.prepare_sino(x, P, cn, O.filter_window(ft, 0.0, P, W, cn))
    assert rel_rmse(q, q_ref) <= 1e-6
    bp = O.bp_compat(q_ref.copy(), O.angle_table(arc, N), c, 1.0, rule="shipped")
    assert np.array_equal(bp.view(np.uint32), sl_ref.view(np.uint32))


@live
def test_sino_repeat_live():
    x = LI.ellipse_sino(9, 90, 128, 1.0, 180.0, n=5, axes=(3.0, 30.0))
    cs = [0.0, 1.5, -3.25, 20.0]
    q_ref, sls = O.lct_sino_repeat(x, cs, O.PHS, 5)
    for k, c in enumerate(cs):
        bp = O.bp_compat(q_ref.copy(), O.angle_table(180.0, 90), c, 1.0, rule="shipped")
        assert np.array_equal(bp.view(np.uint32), sls[k].view(np.uint32)), c


@live
def test_average_gradient_live_in_own_process():
    """AverageGradient reads past a copy it allocates itself; a process of its
    own whose large blocks are fresh zeroed pages makes that read 0."""
    code = (
        "import sys, numpy as np\n"
        f"sys.path[:0] = [{os.path.dirname(HERE)!r}, {GOLD!r}]\n"
        "import oracle as O, lct_inputs as LI\n"
        "O.lct_lib().ref_lct_mmap_threshold(65536)\n"
        "N, W = 241, 160\n"
        "arc = 180.0 * N / (N - 1)\n"
        "p = LI.ellipse_sino(77, N, W, -2.0, arc, n=5, axes=(4.0, 30.0))\n"
        "t = LI.quantise(np.exp(-2 * p / p.max()))\n"
        "axes = np.array([79.5, 78.25, 77.5, 81.0], np.float32)\n"
        "want = O.lct_ag_metric(t, arc, axes)\n"
        "ag = O.AgOracle(t, arc, rule='shipped')\n"
        "got = np.array([ag.apply(a) for a in axes], np.float32)\n"
        "assert np.all(np.abs(got - want) <= 1e-6 * np.abs(want)), (got, want)\n"
        "print('ok')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


def _reference_root():
    p = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "reference_root.txt")
    if not os.path.exists(p):
        return None
    root = open(p).read().strip()
    return root if os.path.isdir(os.path.join(root, "src", "blitz64")) else None


@pytest.mark.skipif(_reference_root() is None, reason="reference Blitz++ headers not here")
def test_cpp_shim_builds_against_blitz():
    """include/ctas_ct.hpp used with blitz::Array<float,2>, as the ct and axis
    tools use CTrec (recr.resize(rec->recShape()), axis.cpp:149)."""
    root = os.path.dirname(HERE)
    ref = os.path.join(root, "oracle", "_ref")
    out = os.path.join(ref, "shim_blitz_check")
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "include"),
                        "-I", os.path.join(ref, "blitz"), "-I", os.path.join(ref, "blitz", "blitz"),
                        "-I", os.path.join(_reference_root(), "src", "blitz64"),
                        os.path.join(HERE, "cpp", "shim_blitz_usage.cpp"),
                        "-L", os.path.join(root, "ctas_b200"), "-lctas_fbp", "-o", out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
