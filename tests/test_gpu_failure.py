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
