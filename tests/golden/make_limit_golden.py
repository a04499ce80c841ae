"""Golden vectors of limit<T> (ctas src/common/external.world.cpp:69-90), the
float -> integer sample conversion of the reference's 8- and 16-bit image
writers, computed by the reference's own template: oracle/Makefile target
`limit` extracts it from external.world.cpp where it lies and builds it with
the reference's flags (oracle/_ref/liblimit_ref.so).

    python tests/golden/make_limit_golden.py

writes tests/golden/limit_ref.npz: the inputs (seeded) and, per case and bits
per sample, the reference's samples.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

BPPS = (8, -8, 16, -16)


def cases():
    """(name, image, mincon, maxcon); mincon == maxcon takes the image's range."""
    rng = np.random.default_rng(20261204)
    noise = rng.standard_normal((64, 96)).astype(np.float32)
    # a fine grid across [0, 1] and beyond, to hit every rounding boundary
    grid = np.linspace(-0.05, 1.05, 64 * 128, dtype=np.float32).reshape(64, 128)
    big = (rng.standard_normal((48, 80)) * 1.0e4 + 3.0e3).astype(np.float32)
    return [
        ("auto_range", noise, 0.0, 0.0),
        ("explicit_range", noise, -0.5, 0.7),
        ("unit_grid", grid, 0.0, 1.0),
        ("large_values", big, -2.0e4, 2.5e4),
        ("constant", np.full((16, 32), 0.25, np.float32), 0.0, 0.0),
    ]


def main():
    import oracle as O
    if not O.ref_limit_available():
        sys.exit("oracle/_ref/liblimit_ref.so is missing: run oracle.build(<ctas checkout>)")
    out = {}
    for name, img, lo, hi in cases():
        out[f"{name}_img"] = img
        out[f"{name}_range"] = np.array([lo, hi], np.float32)
        for bpp in BPPS:
            out[f"{name}_{'s' if bpp < 0 else 'u'}{abs(bpp)}"] = O.ref_limit(img, bpp, lo, hi)
    np.savez_compressed(os.path.join(HERE, "limit_ref.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
