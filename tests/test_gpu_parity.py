"""Parity of the CUDA path with the oracle and the reference's golden outputs.

Bars (written in each test):
* backprojection of a given sinogram (FLT contrast): bit-identical to the
  reference's float arithmetic (golden fixtures from ctas' own ct.cl kernel,
  and the oracle, which those fixtures pin);
* full filter + backprojection: relative RMSE <= 1e-5 and max |diff| <= 1e-4 of
  the image range against the oracle's FP32-compatible path (the FFT is the
  only non-bit-exact step);
* reduced-precision stores: error against the FP64 oracle stated per test.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from ctas_b200 import _lib, ct
from ctas_b200 import phantom as ph

pytestmark = pytest.mark.gpu

# staged backprojection tile ids (7 pixel-tile shapes x 3 arithmetic variants);
# tests/test_host_abi.py checks the library agrees
N_TILES = 21
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def rel_rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b) ** 2)) /
                 max(np.sqrt(np.mean(np.asarray(b, np.float64) ** 2)), 1e-30))


def assert_close_fbp(got, want):
    """relative RMSE <= 1e-5, max abs <= 1e-4 of the image range"""
    want = np.asarray(want, np.float64)
    rng = float(want.max() - want.min()) or 1.0
    assert rel_rmse(got, want) <= 1e-5, rel_rmse(got, want)
    assert float(np.abs(got - want).max()) <= 1e-4 * rng, float(np.abs(got - want).max()) / rng


# --------------------------------------------------------------- golden fixtures
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz"))))
def test_bp_matches_reference_golden_bitexact(path):
    z = np.load(path)
    q = z["q"]
    N, W = q.shape
    arc, c, coeff = float(z["arc"]), float(z["center"]), float(z["coeff"])
    with ct.CTrec((N, W), ct.Contrast.FLT, arc) as rec:
        if coeff != 1.0:
            # recover (pixel size, wavelength) used by the fixture generator
            rec.setPhysics(1.0e-6, 1.0e-10)
            assert ct.rec_cof(1.0e-6, 1.0e-10) == np.float32(coeff)
        out = rec.reconstruct(q.copy(), None, c)
    assert np.array_equal(_bits(out), _bits(z["slice"]))


# --------------------------------------------------------------- BP only (FLT)
@pytest.mark.parametrize("N,W,c,arc", [
    (180, 128, 0.0, 180.0), (181, 127, 3.5, 180.0), (360, 256, -11.75, 180.0),
    (200, 160, 6.25, 360.0), (90, 96, 0.0, 0.5), (720, 512, 0.0, 180.0),
    (1, 8, 0.0, 180.0), (5, 2, 0.0, 180.0), (64, 300, 140.0, 180.0)])
def test_bp_bitexact_vs_oracle(N, W, c, arc):
    rng = np.random.default_rng(N + 7 * W)
    q = rng.standard_normal((N, W)).astype(np.float32)
    tab = O.angle_table(arc, N)
    want = O.bp_compat(q, tab, c, 1.0)
    with ct.CTrec((N, W), ct.Contrast.FLT, arc) as rec:
        got = rec.reconstruct(q.copy(), None, c)
    assert np.array_equal(_bits(got), _bits(want))


def test_bp_explicit_angle_list_bitexact():
    N, W, c = 150, 128, -2.5
    rng = np.random.default_rng(3)
    th = np.sort(rng.uniform(0, np.pi, N))
    q = rng.standard_normal((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, angles=th) as rec:
        got = rec.reconstruct(q.copy(), None, c)
    want = O.bp_compat(q, O.angle_table_list(th), c, 1.0)
    assert np.array_equal(_bits(got), _bits(want))


# --------------------------------------------------------------- full path
@pytest.mark.parametrize("ft,param", [(1, 0.0), (5, 0.0), (6, 0.0), (7, 0.0), (3, 0.0),
                                      (9, 2.0), (10, 0.5), (100, 0.0), (101, 0.0), (0, 0.0)])
def test_full_path_filters(ft, param):
    W, N, c = 200, 240, 1.5
    el = ph.random_ellipses(ft + 11, 6, W, axes=(5, 40))
    s = ph.sinogram(el, N, W, center=c)
    want = O.reconstruct(s, contrast=O.PHS, ftype=ft, fparam=param, center=c)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter(ft, param)) as rec:
        got = rec.reconstruct(s.copy(), None, c)
    assert_close_fbp(got, want)


@pytest.mark.parametrize("W,N,pad", [(512, 720, 0), (64, 90, 0), (100, 64, 0), (255, 100, 0),
                                     (512, 720, 2048), (2560, 24, 4096), (2560, 20, 0),
                                     (33, 40, 64), (4, 3, 0)])
def test_full_path_sizes_and_padding(W, N, pad):
    el = ph.random_ellipses(W + N, 8, W, axes=(2, max(3, W // 5)))
    s = ph.sinogram(el, N, W, center=0.0)
    P = pad or O.padded_width(W)
    want = O.reconstruct(s, contrast=O.PHS, ftype=5, center=0.0, P=P)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), pad=pad) as rec:
        got = rec.reconstruct(s.copy(), None, 0.0)
    assert_close_fbp(got, want)


def test_filtered_sinogram_written_back():
    W, N = 300, 50
    rng = np.random.default_rng(9)
    s = rng.random((N, W)).astype(np.float32)
    P = O.padded_width(W)
    want = O.prepare_sino(s, P, O.PHS, O.filter_window(6, 0.0, P, W, O.PHS))
    x = s.copy()
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HAMMING")) as rec:
        rec.sino(x)
    np.testing.assert_allclose(x, want, rtol=0, atol=2e-6 * np.abs(want).max())
    # NO_WRITEBACK leaves the caller's sinogram alone
    y = s.copy()
    with ct.CTrec((N, W), ct.Contrast.PHS, no_writeback=True) as rec:
        rec.reconstruct(y, None, 0.0)
    assert np.array_equal(y, s)


def test_abs_contrast_and_bad_data():
    W, N, c = 128, 160, -3.0
    el = ph.random_ellipses(5, 5, W, axes=(5, 30))
    p = ph.sinogram(el, N, W, center=c)
    tr = np.exp(-p).astype(np.float32)
    tr[3, 5] = 0.0          # triggers the deAbs clamp (physical.world.cpp:89-98)
    tr[7, 9] = -0.5
    want = O.reconstruct(tr, contrast=O.ABS, ftype=1, center=c)
    with ct.CTrec((N, W), ct.Contrast.ABS) as rec:
        got = rec.reconstruct(tr.copy(), None, c)
        assert_close_fbp(got, want)
        bad = -np.abs(tr) - 1.0
        b0 = bad.copy()
        with pytest.raises(ct.CtasError) as e:
            rec.reconstruct(bad, None, c)
        assert e.value.code == _lib.E_DATA
        assert np.array_equal(bad, b0)    # rejected before any modification


def test_ref_contrast():
    W, N = 128, 100
    rng = np.random.default_rng(4)
    s = (rng.random((N, W)) - 0.5).astype(np.float32)
    want = O.reconstruct(s, contrast=O.REF, ftype=1, center=0.5)
    with ct.CTrec((N, W), ct.Contrast.REF) as rec:
        got = rec.reconstruct(s.copy(), None, 0.5)
    assert_close_fbp(got, want)


def test_physics_coefficient():
    W, N = 96, 120
    rng = np.random.default_rng(8)
    s = rng.random((N, W)).astype(np.float32)
    want = O.reconstruct(s, contrast=O.PHS, ftype=1, center=0.0, pixel_size=6.5e-6,
                         lam=1.2e-10)
    with ct.CTrec((N, W), ct.Contrast.PHS) as rec:
        rec.setPhysics(6.5e-6, 1.2e-10)
        got = rec.reconstruct(s.copy(), None, 0.0)
    assert_close_fbp(got, want)


def test_sino_then_repeat_many_centres():
    # filter once, backproject many centres (CTrec::sino + repeat, lct.cpp:600-646)
    W, N = 160, 180
    el = ph.random_ellipses(21, 5, W, axes=(5, 30))
    s = ph.sinogram(el, N, W)
    with ct.CTrec((N, W), ct.Contrast.PHS) as rec:
        x = s.copy()
        rec.sino(x)
        for c in (-6.5, 0.0, 2.25, 9.0):
            got = rec.repeat(None, c)
            want = O.bp_compat(x, O.angle_table(180.0, N), c, 1.0)
            assert np.array_equal(_bits(got), _bits(want))


def test_errors():
    with ct.CTrec((10, 32), ct.Contrast.PHS) as rec:
        with pytest.raises(ct.CtasError) as e:
            rec.repeat(None, 0.0)
        assert e.value.code == _lib.E_STATE
        with pytest.raises(ct.CtasError) as e:
            rec.reconstruct(np.zeros((10, 32), np.float32), None, 16.0)
        assert e.value.code == _lib.E_CENTER
        with pytest.raises(ct.CtasError) as e:
            rec.reconstruct(np.zeros((10, 31), np.float32), None, 0.0)
        assert e.value.code == _lib.E_SHAPE
        # still usable after errors
        out = rec.reconstruct(np.ones((10, 32), np.float32), None, 0.0)
        assert np.isfinite(out).all()


def test_clone_matches_and_is_independent():
    W, N = 128, 90
    rng = np.random.default_rng(12)
    s = rng.random((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN")) as rec:
        rec.setPhysics(1e-6)
        a = rec.reconstruct(s.copy(), None, 1.0)
        cl = rec.clone()
        b = cl.reconstruct(s.copy(), None, 1.0)
        cl.close()
    assert np.array_equal(_bits(a), _bits(b))


def test_stack_host_and_device_match_single():
    import torch
    W, N, S, c = 192, 120, 7, 2.5
    sinos = np.stack([ph.sinogram(ph.random_ellipses(100 + k, 5, W, axes=(5, 40)), N, W,
                                  center=c) for k in range(S)])
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), chunk_slices=3) as rec:
        singles = np.stack([rec.reconstruct(sinos[k].copy(), None, c) for k in range(S)])
        x = sinos.copy()
        stack = rec.reconstruct_stack(x, None, c)
        assert np.array_equal(_bits(stack), _bits(singles))
        # filtered sinograms written back like the per-slice call does
        y = sinos[2].copy()
        rec.sino(y)
        assert np.array_equal(x[2], y)
        d_in = torch.from_numpy(sinos).cuda()
        d_out = torch.empty((S, W, W), device="cuda")
        rec.reconstruct_stack_dev(d_in, d_out, c)
        torch.cuda.synchronize()
        assert np.array_equal(_bits(d_out.cpu().numpy()), _bits(singles))


def test_device_forms():
    import torch
    W, N, c = 128, 100, -1.25
    rng = np.random.default_rng(1)
    s = rng.random((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.PHS) as rec:
        host = rec.reconstruct(s.copy(), None, c)
        d_s = torch.from_numpy(s).cuda()
        d_o = torch.empty((W, W), device="cuda")
        rec.reconstruct_dev(d_s, d_o, c)
        rec.synchronize()
        assert np.array_equal(_bits(d_o.cpu().numpy()), _bits(host))
        d_f = torch.empty((N, W), device="cuda")
        rec.sino_dev(d_s, d_f)
        rec.repeat_dev(d_o, 3.0)
        torch.cuda.synchronize()
        want = O.bp_compat(d_f.cpu().numpy(), O.angle_table(180.0, N), 3.0, 1.0)
        assert np.array_equal(_bits(d_o.cpu().numpy()), _bits(want))


@pytest.mark.parametrize("store,tol", [(1, 2e-3), (2, 1.5e-2)])
def test_reduced_precision_store(store, tol):
    """FP16 / BF16 filtered sinogram with FP32 accumulation: relative RMSE
    against the FP64 oracle <= tol (FP16 2e-3, BF16 1.5e-2)."""
    W, N, c = 256, 360, 3.5
    el = ph.random_ellipses(77, 8, W, axes=(5, 60))
    s = ph.sinogram(el, N, W, center=c)
    want = O.reconstruct(s, contrast=O.PHS, ftype=5, center=c, fp64=True)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), store=store) as rec:
        got = rec.reconstruct(s.copy(), None, c)
    m = O.mask(W, c)
    assert rel_rmse(got[m], np.asarray(want)[m]) <= tol
    assert (got[~m] == 0).all()


def test_fp32_error_vs_fp64_oracle_is_small():
    W, N, c = 256, 360, 3.5
    el = ph.random_ellipses(78, 8, W, axes=(5, 60))
    s = ph.sinogram(el, N, W, center=c)
    want = O.reconstruct(s, contrast=O.PHS, ftype=5, center=c, fp64=True)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN")) as rec:
        got = rec.reconstruct(s.copy(), None, c)
    assert rel_rmse(got, want) <= 1e-5


def test_cpp_shim_program(tmp_path):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "shim_usage"
    lib_dir = os.path.join(root, "ctas_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "shim_usage.cpp"), "-L", lib_dir,
                    "-lctas_fbp", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    N, W, c = 120, 96, 2.0
    rng = np.random.default_rng(31)
    s = rng.random((N, W)).astype(np.float32)
    s.tofile(tmp_path / "in.f32")
    r = subprocess.run([str(exe), str(N), str(W), str(c), str(tmp_path / "in.f32"),
                        str(tmp_path / "out.f32")], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    out = np.fromfile(tmp_path / "out.f32", np.float32).reshape(2, W, W)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN")) as rec:
        a = rec.reconstruct(s.copy(), None, c)
        b = rec.repeat(None, -c)
    assert np.array_equal(_bits(out[0]), _bits(a))
    assert np.array_equal(_bits(out[1]), _bits(b))


def test_kernel_selection():
    """The staged kernel serves float32 scans of any arc (negative sines through
    the wide layout) once the padded row is 192 columns wide; 16-bit stores
    with negative sines and narrow rows take the generic kernel; all
    bit-exact."""
    rng = np.random.default_rng(2)
    for arc, W, store, want_kernel in ((180.0, 256, 0, 2), (360.0, 256, 0, 2), (180.0, 64, 0, 1),
                                       (360.0, 64, 0, 2), (360.0, 256, 1, 1)):
        N = 120
        q = rng.standard_normal((N, W)).astype(np.float32)
        with ct.CTrec((N, W), ct.Contrast.FLT, arc, store=store) as rec:
            got = rec.reconstruct(q.copy(), None, 1.5)
            assert rec.last_kernel() == want_kernel, (arc, W, store)
        want = O.bp_compat(q, O.angle_table(arc, N), 1.5, 1.0)
        if store == 0:
            assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("tile", list(range(N_TILES)))
@pytest.mark.parametrize("rule", ["ctcl", "shipped"])
def test_wide_layout_every_tile_bitexact(tile, rule):
    """360-degree arcs (negative sines) on the staged kernel: the wide layout's
    halo columns give the reference's flat reads across row ends, and the
    truncating path its rounding toward zero, for every tile and both index
    rules; stack launches included (halos stop at each slice)."""
    N, W, c = 200, 300, -4.25
    rng = np.random.default_rng(100 + tile)
    q = rng.standard_normal((3, N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, 360.0, tile=tile, chunk_slices=3,
                  index_rule=rule) as rec:
        got = rec.reconstruct_stack(q.copy(), None, c)
        assert rec.last_kernel() == 2 and rec.last_tile() == tile
    tab = O.angle_table(360.0, N)
    for s in range(3):
        want = O.bp_compat(q[s], tab, c, 1.0, rule=rule)
        assert np.array_equal(_bits(got[s]), _bits(want)), s


@pytest.mark.parametrize("W,N,c,arc", [(2560, 40, 3.5, 360.0), (512, 181, -60.25, 360.0),
                                       (300, 361, 0.0, 180.0 * 361 / 360), (97, 90, 2.0, 270.0)])
def test_wide_layout_window_checks(W, N, c, arc):
    """Checked staged kernel on the wide layout: every shared-memory gather is
    bounds-checked on the device; no violation, same bits as the oracle."""
    q = np.random.default_rng(W + N).standard_normal((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, arc, checked=True) as rec:
        got = rec.reconstruct(q.copy(), None, c)
        assert rec.last_kernel() == 2
    want = O.bp_compat(q, O.angle_table(arc, N), c, 1.0)
    assert np.array_equal(_bits(got), _bits(want))


def test_wide_layout_filter_and_repeat():
    """Full path on a 360-degree scan: filtered rows written back (halos are
    not part of them), then backprojections at other centres from the kept
    filtered sinogram."""
    N, W = 240, 320
    el = ph.random_ellipses(9, 6, W, axes=(5, 60))
    s = ph.sinogram(el, N, W, center=2.0, arc_deg=360.0)
    with ct.CTrec((N, W), ct.Contrast.PHS, 360.0, ct.Filter("HANN")) as rec:
        x = s.copy()
        got = rec.reconstruct(x, None, 2.0)
        assert rec.last_kernel() == 2
        again = [rec.repeat(None, cc) for cc in (-3.5, 7.25)]
    P = O.padded_width(W)
    q = O.prepare_sino(s, P, O.PHS, O.filter_window(5, 0.0, P, W))
    assert float(np.sqrt(np.mean((x - q) ** 2)) / np.sqrt(np.mean(q ** 2))) <= 1e-5
    tab = O.angle_table(360.0, N)
    assert_close_fbp(got, O.bp_compat(q.astype(np.float64), tab, 2.0, 1.0))
    for cc, g in zip((-3.5, 7.25), again):
        assert_close_fbp(g, O.bp_compat(q.astype(np.float64), tab, cc, 1.0))


@pytest.mark.parametrize("W,N,c", [(2560, 36, 3.5), (1000, 50, -8.0), (513, 720, 0.0)])
def test_fast_kernel_window_checks(W, N, c):
    """Checked variant of the staged kernel: every shared-memory gather is
    bounds-checked on the device; no violation, same bits as the oracle."""
    rng = np.random.default_rng(W)
    q = rng.standard_normal((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, checked=True) as rec:
        got = rec.reconstruct(q.copy(), None, c)
        assert rec.last_kernel() == 2
    want = O.bp_compat(q, O.angle_table(180.0, N), c, 1.0)
    assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("tile", list(range(N_TILES)))
def test_every_tile_bitexact(tile):
    """Every tile configuration of the staged kernel (the autotuner's choices)
    reproduces the reference arithmetic bit for bit, stack launches included."""
    N, W, c = 200, 300, -4.25
    rng = np.random.default_rng(tile)
    q = rng.standard_normal((3, N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, tile=tile, chunk_slices=3) as rec:
        got = rec.reconstruct_stack(q.copy(), None, c)
        assert rec.last_kernel() == 2 and rec.last_tile() == tile
    tab = O.angle_table(180.0, N)
    for s in range(3):
        want = O.bp_compat(q[s], tab, c, 1.0)
        assert np.array_equal(_bits(got[s]), _bits(want))


def test_autotuned_tile_is_reported():
    N, W = 180, 256
    q = np.random.default_rng(5).standard_normal((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT) as rec:
        got = rec.reconstruct(q.copy(), None, 0.0)
        assert 0 <= rec.last_tile() < N_TILES
    assert np.array_equal(_bits(got), _bits(O.bp_compat(q, O.angle_table(180.0, N), 0.0, 1.0)))


@pytest.mark.parametrize("W,N,c,arc,store", [(256, 360, 2.5, 180.0, 0), (96, 120, -1.5, 180.0, 0),
                                             (320, 400, 5.0, 360.0, 0), (256, 300, 0.0, 180.0, 1)])
def test_linear_interpolation_vs_fp64_oracle(W, N, c, arc, store):
    """Linear interpolation (extension): FP32 samples and coordinates against the
    FP64 oracle's linear backprojection of the FP64-filtered sinogram: relative
    RMSE <= 1e-5 (float32 store), <= 2e-3 (float16 store)."""
    el = ph.random_ellipses(W + N, 6, W, axes=(5, W // 5))
    s = ph.sinogram(el, N, W, center=c, arc_deg=arc)
    P = O.padded_width(W)
    qd = O.prepare_sino(s, P, O.PHS, O.filter_window(5, 0.0, P, W, O.PHS, fp64=True), fp64=True)
    want = O.bp_linear(qd, O.angle_table_f64(arc, N), c, 1.0)
    with ct.CTrec((N, W), ct.Contrast.PHS, arc, ct.Filter("HANN"), interp=1, store=store) as rec:
        got = rec.reconstruct(s.copy(), None, c)
        kern = rec.last_kernel()
    assert kern == (2 if W >= 180 else 1)
    m = O.mask(W, c)
    assert rel_rmse(got[m], want[m]) <= (1e-5 if store == 0 else 2e-3)
    assert (got[~m] == 0).all()


def test_uneven_batch_graph_matches_single_calls():
    """Uneven batch (extension): one graph launch (batched filter + persistent
    backprojection) gives the same bits as the per-sinogram loop and as single
    CTrec calls; every slice of the batch."""
    import torch
    rng = np.random.default_rng(17)
    shapes = [(90, 200), (180, 256), (240, 300), (120, 384), (180, 512), (91, 333), (60, 96)]
    jobs, host = [], []
    for k, (N, W) in enumerate(shapes):
        c = float(np.round(rng.uniform(-8, 8), 2))
        el = ph.random_ellipses(300 + k, 5, W, axes=(4, W // 5))
        s = ph.sinogram(el, N, W, center=c)
        host.append((s, c))
        jobs.append((torch.from_numpy(s).cuda(), torch.full((W, W), float("nan"), device="cuda"), c))
    with ct.Batch(jobs, ct.Contrast.PHS, 180.0, ct.Filter("SHEPP-LOGAN")) as b:
        b.run()
        b.synchronize()
        got = [o.cpu().numpy() for _, o, _ in jobs]
        for _, o, _ in jobs:
            o.fill_(float("nan"))
        b.run_loop()
        b.synchronize()
        loop = [o.cpu().numpy() for _, o, _ in jobs]
        assert 0 <= b.tile() < N_TILES
    for k, (N, W) in enumerate(shapes):
        s, c = host[k]
        with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("SHEPP-LOGAN")) as rec:
            single = rec.reconstruct(s.copy(), None, c)
        assert np.array_equal(_bits(got[k]), _bits(single)), k
        assert np.array_equal(_bits(loop[k]), _bits(single)), k


def test_uneven_batch_at_full_size():
    """The 64-sinogram uneven batch at its full size (widths drawn from
    {1024, 1536, 2048, 3072, 4096}, projection counts from {900, 1800, 2400,
    3600}, centres U(-8, 8), Shepp-Logan, random-ellipse phantoms scaled to the
    width): the graph launch equals the per-sinogram launch loop bit for bit for
    all 64, and one sinogram of each width class (plus the largest) matches the
    oracle on sampled rows within the north-star tolerance."""
    import torch
    rng = np.random.default_rng(2026)
    widths, counts = (1024, 1536, 2048, 3072, 4096), (900, 1800, 2400, 3600)
    jobs, meta = [], []
    for k in range(64):
        W = int(rng.choice(widths))
        N = int(rng.choice(counts))
        c = float(rng.uniform(-8, 8))
        el = ph.random_ellipses(7000 + k, 10, W, axes=(5 * W / 512, 120 * W / 512))
        s = ph.sinogram_dev(el[None], N, W, center=c)[0].contiguous()
        jobs.append((s, torch.empty((W, W), device="cuda"), c))
        meta.append((N, W, c, el))
    with ct.Batch(jobs, ct.Contrast.PHS, 180.0, ct.Filter("SHEPP-LOGAN")) as b:
        b.run()
        b.synchronize()
        got = [o.clone() for _, o, _ in jobs]
        b.run_loop()
        b.synchronize()
        for k, (_, o, _) in enumerate(jobs):
            assert torch.equal(got[k], o), k
    picks = {}
    for k, (N, W, c, _) in enumerate(meta):
        picks.setdefault(W, k)
    largest = max(range(64), key=lambda k: meta[k][0] * meta[k][1])
    for k in sorted(set(picks.values()) | {largest}):
        N, W, c, _ = meta[k]
        s = jobs[k][0].cpu().numpy()
        P = O.padded_width(W)
        q = O.prepare_sino(s, P, O.PHS, O.filter_window(100, 0.0, P, W, O.PHS))
        tab = O.angle_table(180.0, N)
        rows = [W // 7, W // 2 - 3, W // 2 + 11, 5 * W // 6]
        want = np.concatenate([O.bp_compat(q, tab, c, 1.0, rows=(r, r + 1)) for r in rows])
        assert_close_fbp(got[k].cpu().numpy()[rows], want)


@pytest.mark.parametrize("R,C,p,sr,sc", [(256, 256, 0.0, 0.0, 0.0), (300, 200, 1.0, 5.0, -3.5),
                                         (400, 400, 0.5, 0.0, 0.0), (150, 180, 0.73, -12.25, 8.0),
                                         (200, 120, 1.5, 0.0, 0.0)])
def test_output_geometry_bitexact(R, C, p, sr, sc):
    """Output geometry (extension): the reference's float mask and index rule at
    the grid's coordinates, bit for bit against the oracle (staged kernel for
    pitches <= 1, generic kernel otherwise); the default grid is the reference's."""
    N, W, c = 180, 256, 2.5
    q = np.random.default_rng(R + C).standard_normal((N, W)).astype(np.float32)
    with ct.CTrec((N, W), ct.Contrast.FLT, out_shape=(R, C), out_pixel=p,
                  out_shift=(sr, sc)) as rec:
        got = rec.reconstruct(q.copy(), None, c)
        kern = rec.last_kernel()
    assert got.shape == (R, C)
    oj, oi, pp = O.geometry(W, R, C, p or 1.0, sr, sc)
    want = O.bp_compat_geom(q, O.angle_table(180.0, N), c, 1.0, R, C, oj, oi, pp)
    assert np.array_equal(_bits(got), _bits(want))
    assert kern == (2 if (p or 1.0) <= 1.0 else 1)
    if (R, C, p) == (256, 256, 0.0):
        assert np.array_equal(_bits(got), _bits(O.bp_compat(q, O.angle_table(180.0, N), c, 1.0)))


@pytest.mark.parametrize("box,W,N", [(3, 256, 120), (10, 300, 91), (1, 64, 40)])
def test_ring_filter(box, W, N):
    """RingFilter::apply (lct.cpp:295-327) before filtering: the corrected
    sinogram written back in FLT contrast is bit-identical to the oracle's;
    the full ring + filter + backprojection path meets the parity tolerance."""
    rng = np.random.default_rng(box + W)
    s = (rng.random((N, W)) + 0.2 * rng.random(W)[None, :]).astype(np.float32)
    want = O.ring(s, box)
    x = s.copy()
    with ct.CTrec((N, W), ct.Contrast.FLT, ring_box=box) as rec:
        rec.sino(x)
    assert np.array_equal(_bits(x), _bits(want))
    full = O.reconstruct(O.ring(s, box), contrast=O.PHS, ftype=5, center=1.5)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), ring_box=box) as rec:
        got = rec.reconstruct(s.copy(), None, 1.5)
    assert_close_fbp(got, full)
