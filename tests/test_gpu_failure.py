"""Failure detection on the GPU without a fault: a bounded device wait that
runs out (an mbarrier nothing arrives at) returns a timeout status, and the
context stays usable -- a reconstruction before and after it agrees bit for
bit.  The pipelined kernels (staged backprojection, tcgen05 convolutions) use
the same bounded try-wait loop with a larger limit."""
import ctypes as C

import numpy as np
import pytest

from ctas_b200 import _lib, ct

pytestmark = pytest.mark.gpu


def _reconstruct():
    rng = np.random.default_rng(3)
    sino = rng.standard_normal((90, 128)).astype(np.float32)
    with ct.CTrec((90, 128), ct.Contrast.PHS, 180.0, ct.Filter("HANN")) as rec:
        out = np.zeros((128, 128), np.float32)
        rec.reconstruct(sino, out, 1.5)
    return out


def test_bounded_wait_times_out_and_context_survives():
    before = _reconstruct()
    L = _lib.load()
    timed_out, seconds = C.c_int32(-1), C.c_double(-1.0)
    _lib.check(L.ctas_probe_bounded_wait(-1, 2000, C.byref(timed_out), C.byref(seconds)))
    assert timed_out.value == 1
    assert 0.0 <= seconds.value < 10.0
    after = _reconstruct()
    assert np.array_equal(before.view(np.uint32), after.view(np.uint32))


def test_bounded_wait_rejects_zero_limit():
    L = _lib.load()
    t, s = C.c_int32(), C.c_double()
    assert L.ctas_probe_bounded_wait(-1, 0, C.byref(t), C.byref(s)) == _lib.E_ARG


@pytest.mark.parametrize("arc,store", [(180.0, 0), (360.0, 0), (180.0, 1)])
def test_staged_kernel_waits_run_out_and_context_survives(arc, store):
    """The production waits of the staged backprojection kernel: with the test
    flag its producer leaves the first chunk of windows uncopied, the
    consumers' and the producer's bounded waits run out, the producer drains
    what it issued, and the call reports CTAS_E_TIMEOUT; a reconstruction
    afterwards equals one before, bit for bit.  (float32, the wide layout of a
    360-degree arc, and the converting 16-bit path.)"""
    N, W = 120, 256
    q = np.random.default_rng(7).standard_normal((N, W)).astype(np.float32)

    def run(flags):
        with ct.CTrec((N, W), ct.Contrast.FLT, arc, store=store, tile=1, flags=flags) as rec:
            return rec.reconstruct(q.copy(), None, 0.5), rec.last_kernel()

    before, k0 = run(0)
    assert k0 == 2
    with pytest.raises(ct.CtasError) as e:
        run(_lib.FLAG_TEST_TIMEOUT)
    assert e.value.code == _lib.E_TIMEOUT
    after, _ = run(0)
    assert np.array_equal(before.view(np.uint32), after.view(np.uint32))


def test_convolution_waits_run_out_and_context_survives():
    """The tcgen05 convolutions' production waits: with the test aid armed each
    kernel's producer leaves its first stage of copies out, the MMA issuer's,
    the epilogue's and the producer's bounded waits run out, the kernel drains
    its copies and MMAs and frees its tensor memory, and the next call reports
    CTAS_E_TIMEOUT; afterwards the same convolutions equal those before, bit
    for bit (weight gradients, whose partial sums are added atomically in any
    order, within 1e-5) -- tiled form, row-streaming form, weight gradient."""
    import torch
    from ctas_b200 import learned
    L = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(5)
    cases = [(64, 128, 1, 16, 32), (32, 32, 1, 16, 128)]  # tiled form, row-streaming form
    data = []
    for cin, cout, B, H, W in cases:
        x = torch.randn((B, H, W, cin), device="cuda", generator=g).bfloat16()
        w = (torch.randn((cout, 9, cin), device="cuda", generator=g) * 0.1).bfloat16()
        dy = torch.randn((B, H, W, cout), device="cuda", generator=g).bfloat16()
        data.append((x, w, dy))

    def run_all():
        outs = []
        for x, w, dy in data:
            outs.append(learned.conv3x3(x, w, None, relu=False).float().cpu())
            dw = torch.zeros(w.shape, dtype=torch.float32, device="cuda")
            learned.conv3x3_wgrad(x, dy, dw)
            outs.append(dw.cpu())
        torch.cuda.synchronize()
        return outs

    before = run_all()

    def armed(fn):
        _lib.check(L.ctas_nn_test_timeout(1))
        try:
            fn()                    # its waits run out on the device
            torch.cuda.synchronize()
        finally:
            _lib.check(L.ctas_nn_test_timeout(0))
        with pytest.raises(ct.CtasError) as e:
            learned.conv3x3(data[0][0], data[0][1], None, relu=False)  # the next call reports it
        assert e.value.code == _lib.E_TIMEOUT
        torch.cuda.synchronize()

    armed(lambda: learned.conv3x3(data[0][0], data[0][1], None, relu=False))   # tiled
    armed(lambda: learned.conv3x3(data[1][0], data[1][1], None, relu=False))   # row-streaming
    armed(lambda: learned.conv3x3_wgrad(data[0][0], data[0][2],
                                        torch.zeros(data[0][1].shape, dtype=torch.float32,
                                                    device="cuda")))           # weight gradient
    after = run_all()
    for k, (a, b) in enumerate(zip(before, after)):
        if k % 2 == 0:
            assert torch.equal(a, b)       # convolution outputs: bit for bit
        else:                              # weight gradients: CTAs add partial sums
            assert torch.allclose(a, b, rtol=1e-5, atol=1e-5 * float(a.abs().max()))
