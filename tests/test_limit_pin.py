"""The oracle's limit<T> (the float -> integer sample conversion of the volume
writers) against the reference's own template, bit for bit.

tests/golden/limit_ref.npz holds outputs of the reference's limit<T>
(ctas src/common/external.world.cpp:69-90), built from the file where it lies
(tests/golden/make_limit_golden.py): an image's own range, an explicit range
with samples beyond it, a fine grid over every rounding boundary, large values,
and a constant image, each as 8- and 16-bit, signed and unsigned samples.  The
device writer (volume.cu) is tested against the oracle in test_gpu_volume.py.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_limit_golden import BPPS, cases  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "limit_ref.npz"))
CASES = cases()


def _key(name, bpp):
    return f"{name}_{'s' if bpp < 0 else 'u'}{abs(bpp)}"


@pytest.mark.parametrize("case", range(len(CASES)), ids=[c[0] for c in CASES])
@pytest.mark.parametrize("bpp", BPPS)
def test_oracle_limit_equals_reference(case, bpp):
    name, img, lo, hi = CASES[case]
    assert np.array_equal(GOLD[f"{name}_img"], img)     # the inputs are the recorded ones
    want = GOLD[_key(name, bpp)]
    got = O.limit(img, bpp, lo, hi)
    assert got.dtype == want.dtype
    assert np.array_equal(got, want)


@pytest.mark.skipif(not O.ref_limit_available(),
                    reason="the reference's limit<T> is built only where its sources are present")
def test_fixtures_are_the_reference_output():
    for name, img, lo, hi in CASES:
        for bpp in BPPS:
            assert np.array_equal(O.ref_limit(img, bpp, lo, hi), GOLD[_key(name, bpp)])
