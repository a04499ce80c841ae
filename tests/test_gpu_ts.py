"""GPU parity of the tomosynthesis step ts_add (ctas src/common/lct.cpp:731-787).

The device filter (a power-of-two FFT of the periodically extended row) and
the oracle's exact FP64 circular convolution agree to float rounding: filtered
rows within 1e-5 of their range (1e-4 with the REF running sum), results
likewise.  The sample index of the projection step is the reference's float
expression on both sides.  A batch of n projections equals n single calls bit
for bit.
"""
import numpy as np
import pytest

import oracle as O
from ctas_b200 import _lib, ct, ts

pytestmark = pytest.mark.gpu


def _case(rows, n, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, n)
    base = 0.6 + 0.3 * np.exp(-(x[None, :] / 0.3) ** 2) * np.cos(3 * x[None, :])
    proj = (base + 0.05 * rng.standard_normal((rows, n))).astype(np.float32)
    res = rng.standard_normal((rows, n)).astype(np.float32)
    return proj, res


@pytest.mark.parametrize("rows,n,cn,ft", [(8, 300, "PHS", "RAMP"), (5, 257, "ABS", "HANN"),
                                          (6, 256, "REF", "RAMP"), (4, 1023, "FLT", "HAMMING"),
                                          (3, 2560, "ABS", "RAMP")])
def test_ts_add_vs_oracle(rows, n, cn, ft):
    proj, res = _case(rows, n, n + rows)
    c, angle, plane = 2.5, 0.35, 7
    contrast = getattr(ct.Contrast, cn)
    fl = ct.Filter(ft)
    want_p, want_r = O.ts_add(proj, res, fl.filter(), 0.0, c, contrast, angle, plane)
    p, r = proj.copy(), res.copy()
    with ts.TS((rows, n), fl, contrast) as t:
        t.add(p, r, c, angle, plane)
    tol = (1e-4 if cn == "REF" else 1e-5) * float(np.ptp(want_p))
    assert float(np.abs(p - want_p).max()) <= tol
    # the result adds one float rounding of its own magnitude
    assert float(np.abs(r - want_r).max()) <= tol + 4 * float(np.spacing(np.abs(want_r).max()))


def test_ts_writeback_off_keeps_projection():
    proj, res = _case(4, 200, 3)
    p = proj.copy()
    with ts.TS((4, 200), ct.Filter("RAMP"), ct.Contrast.ABS) as t:
        t.add(p, res.copy(), 0.0, 0.2, 0, writeback=False)
    assert np.array_equal(p, proj)


def test_ts_batch_equals_sequential_calls():
    import torch
    rows, n, k = 16, 640, 7
    rng = np.random.default_rng(11)
    projs = (0.5 + 0.4 * rng.random((k, rows, n))).astype(np.float32)
    angles = np.linspace(-0.4, 0.4, k).astype(np.float32)
    res0 = rng.standard_normal((rows, n)).astype(np.float32)
    with ts.TS((rows, n), ct.Filter("HANN"), ct.Contrast.ABS) as t:
        P = torch.from_numpy(projs).cuda()
        R = torch.from_numpy(res0).cuda()
        t.add_batch_dev(P, angles, R, 1.25, -4)
        torch.cuda.synchronize()
        got_r, got_p = R.cpu().numpy(), P.cpu().numpy()
        R2 = torch.from_numpy(res0).cuda()
        P2 = torch.from_numpy(projs).cuda()
        for i in range(k):
            t.add_dev(P2[i], R2, 1.25, float(angles[i]), -4)
        torch.cuda.synchronize()
    assert np.array_equal(got_r.view(np.uint32), R2.cpu().numpy().view(np.uint32))
    assert np.array_equal(got_p.view(np.uint32), P2.cpu().numpy().view(np.uint32))


def test_ts_errors():
    with pytest.raises(_lib.CtasError) as e:
        ts.TS((4, 1), ct.Filter("RAMP"), ct.Contrast.PHS)
    assert e.value.code == _lib.E_SHAPE
    with pytest.raises(_lib.CtasError) as e:
        ts.TS((4, 9000), ct.Filter("RAMP"), ct.Contrast.PHS)
    assert e.value.code == _lib.E_UNSUPPORTED
    with pytest.raises(_lib.CtasError) as e:
        ts.TS((4, 64), ct.Filter("KAISER", -1.0), ct.Contrast.PHS)
    assert e.value.code == _lib.E_FILTER


def test_cpp_ts_program(tmp_path):
    """The C++ mirror's ts_add (include/ctas_ct.hpp) over a series equals the
    handle API's sequential adds."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "ts_usage"
    lib_dir = os.path.join(root, "ctas_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "ts_usage.cpp"), "-L", lib_dir,
                    "-lctas_fbp", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    rows, n, k = 6, 333, 4
    imgs = np.stack([_case(rows, n, 40 + i)[0] for i in range(k)])
    imgs.tofile(tmp_path / "in.f32")
    r = subprocess.run([str(exe), str(rows), str(n), str(k), str(tmp_path / "in.f32"),
                        str(tmp_path / "out.f32")], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    got = np.fromfile(tmp_path / "out.f32", np.float32).reshape(rows, n)
    want = np.zeros((rows, n), np.float32)
    with ts.TS((rows, n), ct.Filter("RAMP"), ct.Contrast.ABS) as t:
        for i in range(k):
            angle = np.float32(-0.3) + np.float32(0.6) * np.float32(i) / np.float32(k - 1)
            t.add(imgs[i].copy(), want, 1.5, float(angle), 12)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
