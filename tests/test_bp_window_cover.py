"""CPU proof of the staged backprojector's index bounds (bp_fast.cu).

For every tile and projection, the window the producer fetches must contain
the detector index of every pixel of the tile, and every reconstructed pixel
must read an index in [-1, W] (the padded row's guard columns), for all angle
sets with sin >= 0.  The float32 arithmetic below is the kernel's, operation
for operation (numpy float32 rounds each operation to nearest)."""
import numpy as np
import pytest

import oracle as O

f32 = np.float32
# tile configurations of bp_fast.cu: (rows, cols, window samples)
TILES = [(64, 64, 128), (64, 128, 160), (128, 64, 160), (128, 128, 192), (32, 128, 160)]


def kernel_t(tab, n, jj, ii, W, c):
    sx, cy = f32(tab[2 * n]), f32(tab[2 * n + 1])
    hp = W // 2
    base = f32(c) + (f32(1) - sx - cy) * f32(hp)
    jc = jj.astype(f32) - f32(c)
    return (base + sx * jc) + cy * ii.astype(f32), sx, cy, base


def window_start(sx, cy, base, j0, i0, c, TY, TX, align):
    jc0, jc1 = f32(j0) - f32(c), f32(j0 + TY - 1) - f32(c)
    d0, d1 = cy * f32(i0), cy * f32(i0 + TX - 1)
    b0, b1 = base + sx * jc0, base + sx * jc1
    tmin = min(b0 + d0, b0 + d1, b1 + d0, b1 + d1)
    lo = int(np.floor(tmin)) - 2
    return lo & ~(align - 1)


@pytest.mark.parametrize("W,N,c,angles", [
    (512, 180, 0.0, "uniform"), (256, 360, 3.5, "uniform"), (300, 97, -11.25, "uniform"),
    (2560, 1800, 3.5, "sample"), (4096, 3600, 12.25, "sample"), (1024, 900, 7.9, "sample"),
    (384, 200, 0.0, "random")])
def test_fast_windows_cover_every_pixel(W, N, c, angles):
    if angles == "random":
        th = np.sort(np.random.default_rng(1).uniform(0, np.pi, N))
        tab = O.angle_table_list(th)
        ns = range(N)
    else:
        tab = O.angle_table(180.0, N)
        ns = range(N) if angles == "uniform" else sorted(
            set([0, 1, N // 8, N // 4, N // 3, N // 2, 2 * N // 3, 3 * N // 4, N - 2, N - 1]))
    assert (tab[0::2] >= 0).all()
    m = O.mask(W, c)
    span = ((W + 127) // 128) * 128
    for n in ns:
        jj, ii = np.mgrid[0:span, 0:span]
        t, sx, cy, base = kernel_t(tab, n, jj, ii, W, c)
        k = np.floor(t).astype(np.int64)
        # reconstructed pixels read only [-1, W]; floor == trunc except on (-1, 0)
        km = k[:W, :W][m]
        assert km.min() >= -1 and km.max() <= W
        tt = t[:W, :W][m]
        assert np.array_equal(np.where(tt < 0, 0, np.floor(tt)), np.trunc(tt))
        for TY, TX, BOX in TILES:
            for j0 in range(0, W, TY):
                for i0 in range(0, W, TX):
                    kt = k[j0:j0 + TY, i0:i0 + TX]
                    for align in (4, 8):  # float32 / 16-bit windows
                        x0 = window_start(sx, cy, base, j0, i0, c, TY, TX, align)
                        assert x0 % align == 0
                        assert kt.min() >= x0 and kt.max() < x0 + BOX, \
                            (n, TY, TX, j0, i0, x0, kt.min(), kt.max())


@pytest.mark.parametrize("W,N,c,R,C,p,sr,sc", [
    (512, 90, 3.5, 700, 600, 0.5, 10.0, -20.0), (300, 60, -2.0, 300, 300, 1.0, 7.5, 0.0),
    (256, 120, 0.0, 513, 400, 0.37, 0.0, 0.0)])
def test_fast_windows_cover_output_geometry(W, N, c, R, C, p, sr, sc):
    """Output geometry with pitch <= 1: the window of every tile still holds the
    index of every one of its pixels (coordinates formed as the kernel forms them)."""
    tab = O.angle_table(180.0, N)
    oj, oi, pp = O.geometry(W, R, C, p, sr, sc)
    oj, oi, pp = f32(oj), f32(oi), f32(pp)
    jj_all = oj + pp * np.arange(((R + 127) // 128) * 128, dtype=np.float32)
    ii_all = oi + pp * np.arange(((C + 127) // 128) * 128, dtype=np.float32)
    hp = W // 2
    for n in range(0, N, 7):
        sx, cy = f32(tab[2 * n]), f32(tab[2 * n + 1])
        base = f32(c) + (f32(1) - sx - cy) * f32(hp)
        t = (base + sx * (jj_all[:, None] - f32(c))) + cy * ii_all[None, :]
        k = np.floor(t).astype(np.int64)
        for TY, TX, BOX in TILES:
            for j0 in range(0, R, TY):
                for i0 in range(0, C, TX):
                    kt = k[j0:j0 + TY, i0:i0 + TX]
                    ja, jb = jj_all[j0], jj_all[j0 + TY - 1]
                    ia, ib = ii_all[i0], ii_all[i0 + TX - 1]
                    b0, b1 = base + sx * (ja - f32(c)), base + sx * (jb - f32(c))
                    d0, d1 = cy * ia, cy * ib
                    tmin = min(b0 + d0, b0 + d1, b1 + d0, b1 + d1)
                    for align in (4, 8):
                        x0 = (int(np.floor(tmin)) - 2) & ~(align - 1)
                        assert kt.min() >= x0 and kt.max() < x0 + BOX


def _wide_offset(W):
    return ((W + 16 + 7) // 8) * 8          # fbp_kernels.hpp wide_offset


def _wide_pitch(W):
    return _wide_offset(W) + ((2 * W + 16 + 7) // 8) * 8


@pytest.mark.parametrize("W,N,c,arc,rule", [
    (256, 360, 3.5, 360.0, "ctcl"), (300, 201, -11.25, 360.0, "shipped"),
    (512, 361, 0.0, 180.0 * 361 / 360, "ctcl"), (384, 240, 20.75, 270.0, "shipped"),
    (2560, 3600, 3.5, 360.0, "sample"), (200, 150, -90.25, 360.0, "ctcl"),
    (256, 200, 0.0, "random", "ctcl")])
def test_wide_layout_windows_and_truncation(W, N, c, arc, rule):
    """Angle sets with negative sines (the wide layout): for every tile and
    projection the window holds the index the kernel forms for every pixel of
    the tile; where the tile's corner minimum is below 1 the kernel truncates
    toward zero (ceiling for t < 0), elsewhere it floors, and for every
    reconstructed pixel that equals the reference's truncation; and every index
    read lies inside the wide row (halo columns included)."""
    if arc == "random":
        th = np.sort(np.random.default_rng(3).uniform(0, 2 * np.pi, N))
        tab = O.angle_table_list(th)
        ns = range(0, N, 3)
    else:
        tab = O.angle_table(arc, N)
        ns = range(N) if rule != "sample" else sorted(
            set(list(range(0, N, N // 16)) + [N // 2 - 1, N // 2, N // 2 + 1, N - 1]))
    shipped = rule == "shipped"
    assert (tab[0::2] < 0).any()
    m = O.mask(W, c)
    off, Wp = _wide_offset(W), _wide_pitch(W)
    span = ((W + 127) // 128) * 128
    hp = W // 2
    for n in ns:
        sx, cy = f32(tab[2 * n]), f32(tab[2 * n + 1])
        k0 = f32(1) - (sx + cy) if shipped else (f32(1) - sx) - cy
        base = f32(c) + k0 * f32(hp)
        jj, ii = np.mgrid[0:span, 0:span]
        t = (base + sx * (jj.astype(f32) - f32(c))) + cy * ii.astype(f32)
        fl = np.floor(t).astype(np.int64)
        tr = np.trunc(t).astype(np.int64)
        tm = tr[:W, :W][m]
        assert tm.min() + off >= 0 and tm.max() + off < Wp
        for TY, TX, BOX in TILES:
            for j0 in range(0, W, TY):
                for i0 in range(0, W, TX):
                    jc0, jc1 = f32(j0) - f32(c), f32(j0 + TY - 1) - f32(c)
                    d0, d1 = cy * f32(i0), cy * f32(i0 + TX - 1)
                    b0, b1 = base + sx * jc0, base + sx * jc1
                    tmin = min(b0 + d0, b0 + d1, b1 + d0, b1 + d1)
                    x0 = (int(np.floor(tmin)) - 2) & ~3
                    neg = tmin < f32(1)
                    kt = np.where(t[j0:j0 + TY, i0:i0 + TX] < 0,
                                  np.ceil(t[j0:j0 + TY, i0:i0 + TX]),
                                  fl[j0:j0 + TY, i0:i0 + TX]).astype(np.int64) if neg \
                        else fl[j0:j0 + TY, i0:i0 + TX]
                    assert kt.min() >= x0 and kt.max() < x0 + BOX
                    # a window may start left of the row (pixels outside the
                    # disc; the copy reads 0 there): 16-byte aligned all the same
                    assert ((x0 + off) * 4) % 16 == 0
                    mm = np.zeros((TY, TX), bool)
                    sub_m = m[j0:j0 + TY, i0:i0 + TX]
                    mm[:sub_m.shape[0], :sub_m.shape[1]] = sub_m
                    assert np.array_equal(kt[mm], tr[j0:j0 + TY, i0:i0 + TX][mm]), \
                        (n, TY, TX, j0, i0)
