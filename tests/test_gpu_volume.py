"""GPU tests of the streamed volume call (include/ctas_volume.h): the ct
tool's slice loop (src/executables/ct.cpp:156-206) with read / write
callbacks, raw files, and the writer's sample conversion (limit<T>,
src/common/external.world.cpp:69-90).

The volume call runs the same kernels as the stack call, so its float32
slices must equal the stack call's bit for bit; integer samples must equal
the oracle's restatement of limit<T> applied to those slices, bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ctas_b200 import _lib, ct, volume

pytestmark = pytest.mark.gpu

BPPS = [8, -8, 16, -16, 32, -32, 64, -64]


def _sinos(S, N, W, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(-1, 1, W, dtype=np.float32)
    base = np.maximum(0, 1 - x ** 2)[None, None, :] * rng.uniform(0.5, 2.0, (S, 1, 1))
    return (base + 0.05 * rng.standard_normal((S, N, W))).astype(np.float32)


def _images(shape, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5, 1.5, shape).astype(np.float32)
    flat = x.reshape(shape[0], -1)
    flat[:, :6] = np.float32([0.0, 1.0, 0.5, 0.25, 1.0 - 2 ** -24, 2 ** -24])
    return x


@pytest.mark.parametrize("bpp", BPPS)
@pytest.mark.parametrize("shape", [(3, 64, 96), (2, 37, 5)])   # vector and scalar paths
def test_quantize_fixed_range_matches_oracle(bpp, shape):
    import torch
    x = _images(shape, abs(bpp) + shape[1])
    got = volume.quantize_dev(torch.from_numpy(x).cuda(), bpp, 0.0, 1.0).cpu().numpy()
    for k in range(shape[0]):
        want = O.limit(x[k], bpp, 0.0, 1.0)
        assert got.dtype == want.dtype
        assert np.array_equal(got[k], want), bpp


@pytest.mark.parametrize("bpp", BPPS)
def test_quantize_own_range_matches_oracle(bpp):
    import torch
    x = _images((4, 48, 64), 100 + bpp)
    x[2] = 3.25   # an image of equal values becomes 0
    x[3] *= 1e3
    got = volume.quantize_dev(torch.from_numpy(x).cuda(), bpp).cpu().numpy()
    for k in range(4):
        assert np.array_equal(got[k], O.limit(x[k], bpp)), (bpp, k)
    assert not got[2].any()


def test_quantize_errors():
    import torch
    x = torch.zeros((1, 4, 4), device="cuda")
    with pytest.raises(_lib.CtasError) as e:
        volume.quantize_dev(x, 12)
    assert e.value.code == _lib.E_ARG
    assert _lib.load().ctas_vol_sample_bytes(12) == 0
    assert _lib.load().ctas_vol_sample_bytes(-16) == 2


def _rec(N, W, **kw):
    return ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), no_writeback=True, **kw)


@pytest.mark.parametrize("kw", [dict(chunk_slices=3), dict(chunk_slices=4, ring_box=3),
                                dict(chunk_slices=2, store=1), dict()])
def test_volume_float_equals_stack(kw):
    S, N, W, c = 11, 120, 160, 2.5
    sinos = _sinos(S, N, W, 1)
    with _rec(N, W, **kw) as rec:
        want = rec.reconstruct_stack(sinos.copy(), None, c)
        got = volume.reconstruct_arrays(rec, sinos, c)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("bpp,lo,hi", [(16, 0.0, 0.0), (8, -0.002, 0.01), (-32, 0.0, 0.0),
                                       (-8, -0.01, 0.01), (64, 0.0, 0.0)])
def test_volume_samples_equal_oracle_limit_of_stack(bpp, lo, hi):
    S, N, W, c = 7, 90, 128, -1.5
    sinos = _sinos(S, N, W, 2)
    with _rec(N, W, chunk_slices=3) as rec:
        ref = rec.reconstruct_stack(sinos.copy(), None, c)
        got = volume.reconstruct_arrays(rec, sinos, c, bpp, lo, hi)
    assert got.dtype == volume.sample_dtype(bpp)
    for k in range(S):
        assert np.array_equal(got[k], O.limit(ref[k], bpp, lo, hi)), k


def test_volume_callbacks_in_slice_order_and_chunked():
    S, N, W = 10, 60, 96
    sinos = _sinos(S, N, W, 3)
    reads, writes = [], []
    out = np.zeros((S, W, W), np.float32)

    def read(first, count, buf):
        reads.append((first, count))
        buf[:] = sinos[first:first + count]

    def write(first, count, buf):
        writes.append((first, count))
        out[first:first + count] = buf

    with _rec(N, W, chunk_slices=4) as rec:
        volume.reconstruct_volume(rec, S, 0.0, read, write)
        want = rec.reconstruct_stack(sinos.copy(), None, 0.0)
    assert reads == [(0, 4), (4, 4), (8, 2)]
    assert writes == reads
    assert np.array_equal(out, want)


def test_volume_read_error_ends_call_after_earlier_chunks():
    S, N, W = 12, 60, 96
    sinos = _sinos(S, N, W, 4)
    written = []

    def read(first, count, buf):
        if first >= 6:
            raise ValueError("unreadable sinogram")
        buf[:] = sinos[first:first + count]

    def write(first, count, buf):
        written.append(first)

    with _rec(N, W, chunk_slices=3) as rec:
        with pytest.raises(ValueError, match="unreadable"):
            volume.reconstruct_volume(rec, S, 0.0, read, write)
        assert written == [0, 3]
        # the handle stays usable
        got = volume.reconstruct_arrays(rec, sinos[:2], 0.0)
        assert np.array_equal(got, rec.reconstruct_stack(sinos[:2].copy(), None, 0.0))


def test_volume_write_error_stops_reading():
    S, N, W = 40, 60, 96
    sinos = _sinos(S, N, W, 5)
    reads = []

    def read(first, count, buf):
        reads.append(first)
        buf[:] = sinos[first:first + count]

    def write(first, count, buf):
        raise OSError("disk full")

    with _rec(N, W, chunk_slices=2) as rec:
        with pytest.raises(OSError, match="disk full"):
            volume.reconstruct_volume(rec, S, 0.0, read, write)
    # the reader stopped early: at most the three ring buffers ahead of the
    # four chunks the device took before the failure was seen
    assert len(reads) <= 9, reads


def test_volume_absorption_bad_data():
    """deAbs rejects a slice without positive data (physical.world.cpp:93-94):
    CTAS_E_DATA, the chunks before it written."""
    S, N, W = 9, 40, 64
    sinos = np.abs(_sinos(S, N, W, 6)) + 0.1
    sinos[7] = -1.0
    written = []

    def read(first, count, buf):
        buf[:] = sinos[first:first + count]

    def write(first, count, buf):
        written.append(first)

    rec = ct.CTrec((N, W), ct.Contrast.ABS, 180.0, ct.Filter(), no_writeback=True, chunk_slices=3)
    with rec:
        with pytest.raises(_lib.CtasError) as e:
            volume.reconstruct_volume(rec, S, 0.0, read, write)
    assert e.value.code == _lib.E_DATA
    assert written == [0, 3]


def test_raw_files_roundtrip(tmp_path):
    S, N, W, c = 6, 100, 128, 3.0
    sinos = _sinos(S, N, W, 7)
    fin, fout = tmp_path / "sinos.raw", tmp_path / "rec.raw"
    with open(fin, "wb") as f:
        f.write(b"\0" * 256)            # a header before the dataset
        sinos.tofile(f)
    with _rec(N, W, chunk_slices=4) as rec:
        ref = rec.reconstruct_stack(sinos.copy(), None, c)
        volume.reconstruct_raw(rec, str(fin), S, str(fout), c, -16, in_offset=256, out_offset=64,
                               io_threads=3)
        raw = np.fromfile(fout, np.uint8)
        assert raw.size == 64 + S * W * W * 2
        got = raw[64:].view(np.int16).reshape(S, W, W)
        for k in range(S):
            assert np.array_equal(got[k], O.limit(ref[k], -16))
        # float32 output into a fresh file
        volume.reconstruct_raw(rec, str(fin), S, str(tmp_path / "f.raw"), c, 0, in_offset=256)
        assert np.array_equal(np.fromfile(tmp_path / "f.raw", np.float32).reshape(S, W, W), ref)
        # an input file too short for the request
        with pytest.raises(_lib.CtasError) as e:
            volume.reconstruct_raw(rec, str(fin), S + 1, str(fout), c, 0, in_offset=256)
        assert e.value.code == _lib.E_IO


def test_cpp_volume_usage_program(tmp_path):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "volume_usage"
    lib_dir = os.path.join(root, "ctas_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "volume_usage.cpp"), "-L", lib_dir,
                    "-lctas_fbp", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    S, N, W, c = 5, 90, 128, 1.0
    sinos = _sinos(S, N, W, 8)
    sinos.tofile(tmp_path / "in.f32")
    r = subprocess.run([str(exe), str(S), str(N), str(W), str(c), "8", "0", "0",
                        str(tmp_path / "in.f32"), str(tmp_path / "out.u8")],
                       capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    got = np.fromfile(tmp_path / "out.u8", np.uint8).reshape(S, W, W)
    with ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), no_writeback=True) as rec:
        ref = rec.reconstruct_stack(sinos.copy(), None, c)
    for k in range(S):
        assert np.array_equal(got[k], O.limit(ref[k], 8))
