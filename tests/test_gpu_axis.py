"""GPU parity of the rotation-axis search against the oracle.

Reference: AverageGradient and raxis() (ctas src/common/lct.cpp:792-1297).
The GPU filter is not bit-identical to the oracle's FFT (relative RMSE ~1e-7),
so average-gradient values are compared to a relative 1e-5; on the GPU's own
slice (same filtered data) the metric kernel is compared to 2e-6 (its FP64
separable smoothing versus the oracle's FP64 2-D table).  Search results are
compared to the oracle's search within 1e-3 px, and the number of
reconstructions must match (up to the speculative batch of the directional
march).  Multi-centre backprojection is bit-exact.
"""
import numpy as np
import pytest

import oracle as O
from ctas_b200 import _lib, axis, ct
from ctas_b200 import phantom as ph

pytestmark = pytest.mark.gpu


def _transmission(W, N, c_true, seed, arc=180.0):
    el = ph.random_ellipses(seed, 6, W, axes=(4, max(6, W // 5)))
    p = ph.sinogram(el, N, W, center=c_true, arc_deg=arc)
    return np.exp(-p * (0.7 / max(1e-6, float(p.max())))).astype(np.float32)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("W,N", [(192, 121), (192, 241), (128, 65)])
def test_multi_centre_backprojection_bitexact(W, N):
    """ctas_fbp_repeat_multi_dev == one repeat_dev per centre, staged (W >= 168)
    and generic (W < 168) kernels."""
    import torch
    T = _transmission(W, N, 1.5, 3)
    cs = np.array([0.0, 1.5, -2.25, 7.0, -11.5], np.float32)
    with ct.CTrec((N, W), ct.Contrast.ABS, 180.0, ct.Filter("RAMP"), no_writeback=True) as rec:
        rec.sino(T.copy())
        multi = torch.empty((cs.size, W, W), device="cuda")
        rec.repeat_multi_dev(cs, multi)
        one = torch.empty((W, W), device="cuda")
        for k, c in enumerate(cs):
            rec.repeat_dev(one, float(c))
            torch.cuda.synchronize()
            assert np.array_equal(_bits(multi[k].cpu().numpy()), _bits(one.cpu().numpy()))


@pytest.mark.parametrize("W,N", [(192, 121), (192, 241), (160, 81)])
def test_average_gradient_vs_oracle(W, N):
    T = _transmission(W, N, 2.0, 11)
    ax = np.array([0.5 * (W - 1), 0.5 * (W - 1) + 2.0, 0.5 * (W - 1) - 3.7,
                   0.5 * (W - 1) + 9.0], np.float32)
    with axis.AverageGradient(T, 180.0) as ag:
        got = ag.apply(ax)
        assert abs(ag.sigma - float(O.ag_sigma(180.0, N, W))) <= 1e-6 * ag.sigma
    ora = O.AgOracle(T, 180.0)
    want = np.array([ora.apply(a) for a in ax], np.float32)
    np.testing.assert_allclose(got, want, rtol=1e-5)


def test_average_gradient_kernel_on_same_slice():
    """The smoothing / Sobel / mean kernel against the oracle's metric on the
    GPU's own slice (same filtered data, same backprojection)."""
    import torch
    W, N = 192, 121
    T = _transmission(W, N, -1.0, 5)
    cs = np.array([0.0, -1.0, 3.5], np.float32)
    with ct.CTrec((N, W), ct.Contrast.ABS, 180.0, ct.Filter("RAMP"), no_writeback=True) as rec:
        rec.sino(T.copy())
        sl = torch.empty((cs.size, W, W), device="cuda")
        rec.repeat_multi_dev(cs, sl)
        torch.cuda.synchronize()
        slices = sl.cpu().numpy()
    with axis.AverageGradient(T, 180.0) as ag:
        got = ag.apply(cs + np.float32(0.5 * (W - 1)))
        sigma = ag.sigma
    for k, c in enumerate(cs):
        want = O.ag_metric(slices[k], c, sigma)[0]
        assert abs(float(got[k]) - float(want)) <= 2e-6 * abs(float(want))


@pytest.mark.parametrize("algo", [0, 1, 2, 3])
@pytest.mark.parametrize("W,N,c_true,max_dev", [(192, 121, 2.0, 0.05), (176, 177, -3.0, 0.1)])
def test_raxis_matches_oracle(algo, W, N, c_true, max_dev):
    T = _transmission(W, N, c_true, 21)
    # algo 2/3 start from estimates that must lie within max_dev
    try:
        want, want_calls = O.raxis(T, 180.0, max_dev, algo)
    except ValueError as e:
        with pytest.raises(_lib.CtasError):
            axis.raxis(T, 180.0, max_dev, algo)
        return
    got, calls = axis.raxis(T, 180.0, max_dev, algo, return_trials=True)
    assert abs(got - float(want)) <= 1e-3, (got, want)
    assert calls == want_calls
    if algo:
        assert abs(got - (0.5 * (W - 1) + c_true)) <= 1.5


def test_raxis_no_local_minimum_marches_outwards():
    """An axis outside the grid of trials: the directional search (exec2)."""
    W, N, c_true = 192, 121, 12.0  # grid -8, 0, +8 (max_dev 0.05): minimum beyond it
    T = _transmission(W, N, c_true, 8)
    want, want_calls = O.raxis(T, 180.0, 0.05, 1)
    got, calls = axis.raxis(T, 180.0, 0.05, 1, return_trials=True)
    assert abs(got - float(want)) <= 1e-3
    # the march is evaluated in speculative batches of 8: at most 7 extra
    assert want_calls <= calls <= want_calls + 7


@pytest.mark.parametrize("a", [127.5, 131.0, 118.25])
def test_raxis_pair_matches_oracle(a):
    W, rows = 256, 3
    x = np.arange(W, dtype=np.float64)
    f = lambda t: 1.0 + 0.5 * np.exp(-((t - 90) / 12) ** 2) + 0.3 * np.exp(-((t - 170) / 20) ** 2)
    p0 = np.tile(f(x), (rows, 1)).astype(np.float32)
    p180 = np.tile(f(2 * a - x), (rows, 1)).astype(np.float32)
    want = O.raxis_pair(p0, p180, 0.1)
    got = axis.raxis_pair(p0, p180, 0.1)
    assert abs(got - float(want)) <= 1e-3


def test_axis_errors():
    T = _transmission(64, 33, 0.0, 1)
    with pytest.raises(_lib.CtasError) as e:
        axis.raxis(T[:2], 180.0, 0.1, 1)
    assert e.value.code == _lib.E_SHAPE
    with pytest.raises(_lib.CtasError) as e:
        axis.raxis(T, 90.0, 0.1, 1)          # arc below 180 degrees
    assert e.value.code == _lib.E_ARG
    with pytest.raises(_lib.CtasError) as e:
        axis.raxis(T, 180.0, 0.3, 1)         # max_dev above 0.25
    assert e.value.code == _lib.E_ARG
    with pytest.raises(_lib.CtasError) as e:
        axis.raxis(T, 180.0, 0.1, 7)
    assert e.value.code == _lib.E_ARG
    z = np.ones((2, 64), np.float32)         # |p - 1| sums to zero
    with pytest.raises(_lib.CtasError) as e:
        axis.raxis_pair(z, z, 0.1)
    assert e.value.code == _lib.E_DATA
    with pytest.raises(_lib.CtasError) as e:
        axis.AverageGradient(np.zeros((0, 64), np.float32))
    assert e.value.code == _lib.E_SHAPE


def test_cpp_axis_program(tmp_path):
    """The C++ mirror (include/ctas_ct.hpp) gives the Python API's results."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "axis_usage"
    lib_dir = os.path.join(root, "ctas_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "axis_usage.cpp"), "-L", lib_dir,
                    "-lctas_fbp", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    W, N = 176, 177
    T = _transmission(W, N, -3.0, 21)
    T.tofile(tmp_path / "in.f32")
    r = subprocess.run([str(exe), str(N), str(W), "0.1", str(tmp_path / "in.f32")],
                       capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    vals = r.stdout.split()
    for algo in range(4):
        if vals[algo] == "err":
            with pytest.raises(_lib.CtasError):
                axis.raxis(T, 180.0, 0.1, algo)
        else:
            assert abs(float(vals[algo]) - axis.raxis(T, 180.0, 0.1, algo)) <= 1e-4
    with axis.AverageGradient(T, 180.0) as ag:
        assert abs(float(vals[4]) - float(ag.apply(0.5 * (W - 1)))) <= 1e-6 * abs(float(vals[4]))
