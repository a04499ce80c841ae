"""Generate the golden backprojection fixtures from the reference's own kernel.

Each fixture bp_*.npz holds a seeded input (a float32 N x W sinogram `q`,
treated as already filtered), the angle table the reference builds for it
(lct.cpp:512-517), the centre and physics coefficient, and the slice that the
reference's OpenCL kernel `fbp` (ctas src/common/ct.cl:5-44) produces for it,
run on the host through oracle/_ref (see oracle/Makefile).  The fixtures pin
the oracle and the CUDA backprojector bit for bit on machines where the
reference sources are absent.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

CASES = [
    # name, N, W, centre, arc (deg), physics (pixel size m, wavelength m), input kind
    ("basic", 90, 64, 0.0, 180.0, (0.0, 0.0), "normal"),
    ("odd_width", 91, 65, 3.5, 180.0, (0.0, 0.0), "normal"),
    ("arc360_flat_reads", 120, 96, -7.25, 360.0, (0.0, 0.0), "normal"),
    ("step_arc", 60, 48, 2.0, 0.5, (0.0, 0.0), "normal"),
    ("physics", 180, 128, 12.25, 180.0, (1.0e-6, 1.0e-10), "normal"),
    ("near_max_centre", 45, 40, -15.5, 180.0, (0.0, 0.0), "normal"),
    ("tiny", 1, 4, 0.0, 180.0, (0.0, 0.0), "normal"),
    ("smooth", 200, 192, 0.5, 180.0, (0.0, 0.0), "smooth"),
]


def make_input(kind, N, W, seed):
    rng = np.random.default_rng(seed)
    if kind == "smooth":
        k = np.arange(W) - W / 2
        base = np.exp(-(k / (0.3 * W)) ** 2)
        return (base[None, :] * (1 + 0.1 * np.sin(np.arange(N) / 7.0))[:, None]
                + 0.01 * rng.standard_normal((N, W))).astype(np.float32)
    return rng.standard_normal((N, W)).astype(np.float32)


def main():
    if not O.ref_available():
        O.build()  # needs CTAS_REFERENCE_ROOT
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for idx, (name, N, W, c, arc, phys, kind) in enumerate(CASES):
        q = make_input(kind, N, W, 1000 + idx)
        tab = O.angle_table(arc, N)
        coeff = O.rec_cof(*phys) if phys != (0.0, 0.0) else 1.0
        sl = O.ref_fbp(q, tab, c, coeff, nthreads=4)
        np.savez_compressed(os.path.join(out_dir, f"bp_{name}.npz"), q=q, tab=tab,
                            center=np.float32(c), arc=np.float32(arc),
                            coeff=np.float32(coeff), slice=sl)
        print(name, N, W, c, arc, coeff, float(np.abs(sl).max()))


if __name__ == "__main__":
    main()
