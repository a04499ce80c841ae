"""The oracle's restatement of the volume writer's sample conversion,
limit<T> (src/common/external.world.cpp:69-90), pinned by known answers
worked out by hand from the reference's float operations (the reference's
writer needs HDF5 / libtiff / Magick++ and is not built here)."""
import numpy as np
import pytest

import oracle as O


def test_unsigned_8_known_answers():
    x = np.float32([0.0, 0.5, 1.0, -0.1, 1.2, 0.25, 0.999999, 0.002])
    # 0.5 * 255 = 127.5 -> 127; 0.25 * 255 = 63.75 -> 63; 0.999999 * 255 = 254.99975 -> 254
    # 0.002 * 255 = 0.51 -> 0
    assert O.limit(x, 8, 0.0, 1.0).tolist() == [0, 127, 255, 0, 255, 63, 254, 0]


def test_signed_8_truncates_toward_zero():
    x = np.float32([0.0, 0.5, 1.0, 0.25, 0.75])
    # -128 + 127.5 = -0.5 -> 0; -128 + 63.75 = -64.25 -> -64; -128 + 191.25 = 63.25 -> 63
    assert O.limit(x, -8, 0.0, 1.0).tolist() == [-128, 0, 127, -64, 63]


def test_sixteen_bit_known_answers():
    x = np.float32([0.5, 0.25, 1.0])
    assert O.limit(x, 16, 0.0, 1.0).tolist() == [32767, 16383, 65535]
    assert O.limit(x, -16, 0.0, 1.0).tolist() == [0, -16384, 32767]


def test_wide_types_saturate_at_the_top():
    # float(UINT32_MAX) - 0 rounds to 2^32: interim 1 would be 2^32, undefined
    # in C++; the restatement saturates
    x = np.float32([1.0, 0.5])
    assert O.limit(x, 32, 0.0, 1.0).tolist() == [2 ** 32 - 1, 2 ** 31]
    assert O.limit(x, -32, 0.0, 1.0).tolist() == [2 ** 31 - 1, 0]
    assert O.limit(x, 64, 0.0, 1.0).tolist() == [2 ** 64 - 1, 2 ** 63]
    assert O.limit(x, -64, 0.0, 1.0).tolist() == [2 ** 63 - 1, 0]


def test_own_range_and_flat_image():
    x = np.float32([[2.0, 4.0], [3.0, 6.0]])
    # range (2, 6): (3 - 2) / 4 * 255 = 63.75 -> 63; (4 - 2) / 4 * 255 = 127.5 -> 127
    assert O.limit(x, 8).tolist() == [[0, 127], [63, 255]]
    assert not O.limit(np.full((3, 3), 7.5, np.float32), 16).any()
    assert not O.limit(np.full((3, 3), 7.5, np.float32), -8).any()   # 0, not the minimum


def test_range_order_of_operations():
    """(v - min) / (max - min) in float, then the product and the sum, each
    rounded once: agrees with a numpy float32 restatement element for element."""
    rng = np.random.default_rng(0)
    x = rng.uniform(-3, 7, 5000).astype(np.float32)
    lo, hi = np.float32(-1.3), np.float32(5.7)
    interim = (x - lo) / (hi - lo)
    for bpp, dt in ((8, np.uint8), (-8, np.int8), (16, np.uint16), (-16, np.int16)):
        info = np.iinfo(dt)
        tw = np.float32(info.max) - np.float32(info.min)
        v = np.float32(info.min) + interim * tw
        want = np.where(interim < 0, info.min, np.where(interim > 1, info.max, np.trunc(v)))
        assert np.array_equal(O.limit(x, bpp, lo, hi), want.astype(dt)), bpp


def test_bad_bpp():
    with pytest.raises(KeyError):
        O.limit(np.zeros(3, np.float32), 12)
