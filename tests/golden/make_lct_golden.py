"""Generate the lct_*.npz fixtures from the reference's own reconstruction code.

The reference's src/common/lct.cpp (with the library files it needs) is built
in place as shipped (-ffast-math, no -O) by oracle/Makefile into
oracle/_ref/liblct_shipped.so; this script runs CTrec::reconstruct, sino +
repeat, RingFilter::apply, ts_add, raxis and AverageGradient through it and
stores inputs (or their SHA-256 where the tests regenerate them), parameters
and outputs.  Large cases keep sampled rows only.

Run from the repository root, with the reference tree at hand:
    CTAS_REFERENCE_ROOT=<ctas checkout> python tests/golden/make_lct_golden.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
import oracle as O  # noqa: E402
import lct_inputs as LI  # noqa: E402

PHS, REF, ABS, FLT = O.PHS, O.REF, O.ABS, O.FLT
RAMP, WELCH, PARZEN, HANN, HAMMING, BLACKMAN, LANCKZOS, KAISER, GAUSS = 1, 3, 4, 5, 6, 7, 8, 9, 10

# name: (input kind, N, W, contrast, ftype, fparam, arc, centre, pixel size, lambda,
#        keep every k-th slice row (0 = all rows, input stored))
FULL = {
    "phs_hann": ("ell", 180, 192, PHS, HANN, 0.0, 180.0, 2.5, 0.0, 0.0),
    "ref_ramp": ("ell", 120, 128, REF, RAMP, 0.0, 180.0, -1.5, 0.0, 0.0),
    "abs_clamp": ("trans", 90, 160, ABS, HAMMING, 0.0, 180.0, 0.5, 0.0, 0.0),
    "flt": ("normal", 60, 96, FLT, RAMP, 0.0, 180.0, 3.0, 0.0, 0.0),
    "step_physics": ("ell", 100, 128, PHS, WELCH, 0.0, 0.75, 4.25, 1.5e-6, 1e-10),
    "arc360": ("ell", 150, 128, PHS, BLACKMAN, 0.0, 360.0, -3.5, 0.0, 0.0),
    "kaiser": ("ell", 90, 128, PHS, KAISER, 3.0, 180.0, 0.0, 0.0, 0.0),
    "gauss": ("ell", 90, 128, PHS, GAUSS, 0.4, 180.0, -0.75, 0.0, 0.0),
    "parzen": ("ell", 90, 128, PHS, PARZEN, 0.0, 180.0, 1.0, 0.0, 0.0),
    "lanckzos": ("ell", 90, 130, PHS, LANCKZOS, 0.0, 180.0, 2.0, 0.0, 0.0),
}
# large cases: (N, W, contrast, ftype, centre, photons, seed, n ellipses, row stride)
LARGE = {
    # one slice of the 1800 x 2560 Hann stack, reference padding 8192, noise 1e4
    "c1_rows": (1800, 2560, PHS, HANN, 3.5, 1e4, 21, 30, 160),
    # one slice of the 512-wide RAMP case (720 projections, padding 1024, centre 255.5)
    "c0": (720, 512, PHS, RAMP, 0.0, 0.0, 20, 10, 4),
    # a 4096-wide Hamming slice at centre +12.25 (padding 8192), 360 projections
    "c4_rows": (360, 4096, PHS, HAMMING, 12.25, 5e3, 24, 30, 256),
    # a 3072-wide Ramp slice (padding 8192), centre -5.3
    "c2_rows": (300, 3072, PHS, RAMP, -5.3, 0.0, 22, 10, 192),
}


def full_input(kind, seed, N, W, c, arc):
    if kind == "ell":
        return LI.ellipse_sino(seed, N, W, c, arc, n=8, axes=(5.0, W / 4.0))
    if kind == "trans":
        return LI.transmission(seed, N, W, c)
    return LI.normal(seed, N, W)


def main():
    if not O.lct_available("shipped"):
        O.build()
    out = {}
    for k, (name, (kind, N, W, cn, ft, fp, arc, c, ps, lam)) in enumerate(FULL.items()):
        x = full_input(kind, 100 + k, N, W, c, arc)
        q, sl = O.lct_reconstruct(x, cn, ft, fp, arc, c, ps, lam)
        out[f"lct_{name}.npz"] = dict(sino=x, filtered=q, slice=sl, contrast=cn, ftype=ft,
                                      fparam=np.float32(fp), arc=np.float32(arc),
                                      center=np.float32(c), pixel_size=np.float32(ps),
                                      lam=np.float32(lam))
        print(name, N, W, float(np.abs(sl).max()), flush=True)
    for name, (N, W, cn, ft, c, photons, seed, nel, stride) in LARGE.items():
        x = LI.ellipse_sino(seed, N, W, c, 180.0, n=nel, axes=(5.0, 0.23 * W),
                            rho=(0.05, 0.5) if nel == 30 else (0.1, 1.0), photons=photons)
        q, sl = O.lct_reconstruct(x, cn, ft, 0.0, 180.0, c)
        rows = np.arange(0, W, stride)
        qrows = np.linspace(0, N - 1, 16).astype(np.int64)
        out[f"lct_{name}.npz"] = dict(sino_sha=LI.sha(x), N=N, W=W, photons=photons, seed=seed,
                                      n_ellipses=nel, rows=rows, slice_rows=sl[rows],
                                      filtered_rows_idx=qrows, filtered_rows=q[qrows],
                                      contrast=cn, ftype=ft, fparam=np.float32(0.0),
                                      arc=np.float32(180.0), center=np.float32(c),
                                      pixel_size=np.float32(0.0), lam=np.float32(0.0))
        print(name, N, W, float(np.abs(sl).max()), flush=True)
    # windows: Filter::fill (lct.cpp:122-209) per filter and length
    specs = [(0, 0.0), (1, 0.0), (2, 0.0), (3, 0.0), (4, 0.0), (5, 0.0), (6, 0.0), (7, 0.0),
             (8, 0.0), (9, 3.0), (9, 0.5), (10, 0.4), (10, 2.0)]
    wins = {}
    for P in (16, 1024, 4096):
        for ft, fp in specs:
            wins[f"w_{P}_{ft}_{fp:g}"] = O.lct_filter_fill(ft, fp, P)
    for ft in (1, 5, 6):
        wins[f"w_8192_{ft}_0"] = O.lct_filter_fill(ft, 0.0, 8192)
    out["lct_windows.npz"] = wins
    # RingFilter::apply (lct.cpp:295-327)
    x = LI.normal(300, 120, 160)
    out["lct_ring.npz"] = dict(sino_sha=LI.sha(x), **{f"box{b}": O.lct_ring(x, b) for b in (1, 3, 7)})
    # ts_add (lct.cpp:739-787), three projections accumulated
    p = LI.quantise(np.random.default_rng(301).uniform(0.2, 1.0, (40, 200)))
    res = np.zeros((40, 200), np.float32)
    ts = dict(proj=p)
    for k, (ft, c, cn, ang, plane) in enumerate([(RAMP, 0.0, PHS, 0.3, 10),
                                                 (HANN, 2.5, REF, -0.2, -5),
                                                 (HAMMING, -1.5, ABS, 0.1, 3)]):
        fp_, res = O.lct_ts_add(p, res, ft, 0.0, c, cn, ang, plane)
        ts[f"filtered{k}"] = fp_
        ts[f"result{k}"] = res
    out["lct_ts.npz"] = ts
    # raxis algorithm 0 (projection pairs, lct.cpp:1217-1297)
    rax = {}
    for k, true_c in enumerate((0.0, 3.0, -5.5)):
        x = LI.ellipse_sino(310 + k, 361, 192, true_c, 180.0 * 361 / 360, n=8, axes=(5.0, 50.0))
        rax[f"sino_sha{k}"] = LI.sha(x)
        rax[f"axis{k}"] = np.float32(O.lct_raxis(x, 180.0 * 361 / 360, 0.1, 0))
    out["lct_raxis0.npz"] = rax
    # AverageGradient metric (lct.cpp:804-915), in a process of its own
    subprocess.run([sys.executable, os.path.join(HERE, "make_lct_golden.py"), "--ag"], check=True)
    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, name), **d)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name)))


def ag_metric_fixture():
    """AverageGradient values with and without the Gaussian smoothing; the
    reference's read past its own sinogram copy sees fresh zeroed pages here."""
    O.lct_lib().ref_lct_mmap_threshold(65536)
    d = {}
    for k, (N, W) in enumerate(((361, 192), (181, 512), (121, 300))):
        arc = 180.0 * N / (N - 1)
        p = LI.ellipse_sino(320 + k, N, W, 1.0, arc, n=6, axes=(5.0, W / 8.0))
        t = LI.quantise(np.exp(-2.0 * p / float(p.max())))
        axes = np.array([W / 2 - 0.5, W / 2 + 0.5, W / 2 + 1.75, W / 2 - 3.25, W / 2 + 6.0],
                        np.float32)
        d[f"trans{k}"] = t
        d[f"arc{k}"] = np.float32(arc)
        d[f"axes{k}"] = axes
        d[f"metric{k}"] = O.lct_ag_metric(t, arc, axes)
    np.savez_compressed(os.path.join(HERE, "lct_agmetric.npz"), **d)
    print("wrote lct_agmetric.npz")


if __name__ == "__main__":
    if "--ag" in sys.argv:
        ag_metric_fixture()
    else:
        main()
