"""ctas_fbp_reconstruct_dev_noalloc: the entry point for callers that cannot
allocate device memory (frameworks that own every device allocation, fixed
memory budgets, plug-ins).  It keeps its scratch in one fixed array inside the
library, so these tests check that two calls in a row -- of different shapes,
the second reusing what the first left in the array -- give what the handle
path gives, within the parity tolerance of the other tests (relative RMSE
<= 1e-5, max |diff| <= 1e-4 of the image range), and that sizes beyond the
array are refused with a clear error.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

from ctas_b200 import _lib, ct
from ctas_b200 import phantom as ph

pytestmark = pytest.mark.gpu


def _noalloc(sino, slice_, N, W, contrast, ftype, fparam, arc, pad, center, ps=0.0, lam=0.0):
    import torch
    L = _lib.load()
    rc = L.ctas_fbp_reconstruct_dev_noalloc(
        C.c_void_p(sino.data_ptr()), C.c_void_p(slice_.data_ptr()), N, W, contrast, ftype,
        fparam, arc, pad, center, ps, lam, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


def _close(got, want):
    want = want.astype(np.float64)
    rng = float(want.max() - want.min()) or 1.0
    rmse = np.sqrt(np.mean((got - want) ** 2)) / max(np.sqrt(np.mean(want ** 2)), 1e-30)
    assert rmse <= 1e-5, rmse
    assert np.abs(got - want).max() <= 1e-4 * rng


def test_noalloc_two_calls_match_handle_path():
    import torch
    cases = [  # first call larger than the second: leftovers must not leak
        dict(N=720, W=512, contrast=ct.Contrast.PHS, ftype=5, fparam=0.0, arc=180.0, pad=0,
             center=2.5, ps=1e-6, lam=0.0),
        dict(N=500, W=384, contrast=ct.Contrast.REF, ftype=1, fparam=0.0, arc=180.0, pad=2048,
             center=-3.0, ps=0.0, lam=0.0),
        # a 360-degree arc has negative sines: the one-pixel-per-thread kernel
        dict(N=400, W=128, contrast=ct.Contrast.PHS, ftype=6, fparam=0.0, arc=360.0, pad=0,
             center=1.5, ps=0.0, lam=0.0),
    ]
    for k, cs in enumerate(cases):
        N, W = cs["N"], cs["W"]
        el = ph.random_ellipses(40 + k, 6, W, axes=(5, W // 6))
        s = torch.from_numpy(ph.sinogram(el, N, W, center=cs["center"])).cuda()
        out = torch.full((W, W), float("nan"), device="cuda")
        rc = _noalloc(s, out, N, W, cs["contrast"], cs["ftype"], cs["fparam"], cs["arc"],
                      cs["pad"], cs["center"], cs["ps"], cs["lam"])
        assert rc == 0, _lib.load().ctas_fbp_last_error()
        torch.cuda.synchronize()
        with ct.CTrec((N, W), cs["contrast"], cs["arc"], ct.Filter(cs["ftype"], cs["fparam"]),
                      pad=cs["pad"]) as rec:
            rec.setPhysics(cs["ps"], cs["lam"])
            want = torch.empty((W, W), device="cuda")
            rec.reconstruct_dev(s, want, cs["center"])
            rec.synchronize()
        _close(out.cpu().numpy(), want.cpu().numpy())


def test_noalloc_refuses_sizes_beyond_its_scratch():
    import torch
    N, W = 1800, 8192                      # 59 MB of filtered rows > 32 MiB
    s = torch.zeros((4, 4), device="cuda")  # never read: the size check comes first
    rc = _noalloc(s, s, N, W, ct.Contrast.PHS, 1, 0.0, 180.0, 0, 0.0)
    assert rc == _lib.E_SHAPE
    msg = _lib.load().ctas_fbp_last_error().decode()
    assert "32 MiB" in msg and "1800 x 8192" in msg


def test_noalloc_allocates_nothing():
    """Once every kernel has run once, further calls of every shape leave the
    device's free memory and torch's allocator untouched."""
    import torch
    shapes = [(720, 512, 2.5), (400, 128, -1.5), (1000, 1024, 4.0)]
    bufs = []
    for k, (N, W, c) in enumerate(shapes):
        el = ph.random_ellipses(60 + k, 5, W, axes=(5, W // 6))
        s = torch.from_numpy(ph.sinogram(el, N, W, center=c)).cuda()
        bufs.append((s, torch.empty((W, W), device="cuda"), N, W, c))
    torch.cuda.synchronize()
    # one call of each shape first: lazy module loading may place kernel code
    # in device memory on a kernel's first launch
    for s, out, N, W, c in bufs:
        assert _noalloc(s, out, N, W, ct.Contrast.PHS, 5, 0.0, 180.0, 0, c) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    alloc0 = torch.cuda.memory_allocated()
    for s, out, N, W, c in bufs[::-1] + bufs:
        rc = _noalloc(s, out, N, W, ct.Contrast.PHS, 5, 0.0, 180.0, 0, c)
        assert rc == 0, _lib.load().ctas_fbp_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_refuses_a_capturing_stream():
    import torch
    N, W = 180, 256
    s = torch.zeros((N, W), device="cuda")
    out = torch.zeros((W, W), device="cuda")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out.add_(1.0)                       # the graph holds one op of its own
        rc = _noalloc(s, out, N, W, ct.Contrast.PHS, 1, 0.0, 180.0, 0, 0.0)
    assert rc == _lib.E_ARG
    assert b"capturing" in _lib.load().ctas_fbp_last_error()
