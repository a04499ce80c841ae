"""The roofline arithmetic of bench.py, recomputed independently (CPU only):
nominal shared-memory peak, in-mask update bytes, the staged kernel's TMA window
bytes for its tile shape, and the filter's shared-memory passes."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402
import oracle as O  # noqa: E402
from ctas_b200 import ct  # noqa: E402


def test_roofline_fields():
    bp_ms, S, f_ms, sms, mhz = 200.0, 128, 4.0, 148, 1965.0
    r = bench.roofline(bp_ms, S, f_ms, 36000.0, {"sm_mhz": mhz}, sms, 16000.0, 15)
    nominal = 128.0 * sms * mhz * 1e6 / 1e9
    assert abs(r["peak"] - round(nominal, 1)) < 1e-6
    inmask = int(O.mask(bench.WIDTH, bench.CENTER).sum())
    bp_bytes = 4.0 * bench.N_ANGLES * inmask * S
    assert r["algorithmic_bytes_per_launch"] == bp_bytes
    assert abs(r["achieved"] - bp_bytes / (bp_ms * 1e-3) / 1e9) < 0.1
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    assert abs(r["probe"]["frac"] - r["achieved"] / 36000.0) < 1e-3

    # windows: one BOX-sample copy per projection for every tile touching the disc
    ty, tx, box = ct.tile_shape(15)
    assert (ty, tx, box) == (64, 128, 160)
    m = O.mask(bench.WIDTH, bench.CENTER)
    active = 0
    for j0 in range(0, bench.WIDTH, ty):
        for i0 in range(0, bench.WIDTH, tx):
            active += bool(m[j0:j0 + ty, i0:i0 + tx].any())
    assert r["l2_windows"]["window_bytes_per_launch"] == 4.0 * box * bench.N_ANGLES * active * S

    # filter: 4 ns - 4 passes over PAD complex floats per row pair
    ns = {4096: 4, 8192: 5}[bench.PAD]
    want = ((bench.N_ANGLES + 1) // 2) * (4 * ns - 4) * bench.PAD * 8.0 * S
    assert r["filter"]["smem_passes"]["bytes_per_launch"] == want
    assert np.isclose(r["filter"]["achieved"],
                      4.0 * bench.N_ANGLES * bench.WIDTH * 2 * S / (f_ms * 1e-3) / 1e9, atol=0.1)
