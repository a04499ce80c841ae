"""Streamed volume reconstruction: Python face of include/ctas_volume.h.

The ct tool's slice loop (src/executables/ct.cpp:156-206 -- read a sinogram,
ring-filter, reconstruct, save the slice) as one pipelined call on a
``CTrec``: a reader callback fills a pinned input ring, the device filters
and backprojects chunk after chunk with both copy directions overlapped, and
a writer callback receives the slices -- float32, or integer samples
converted on the device as the reference's ``limit<T>`` does
(src/common/external.world.cpp:69-90; the ct tool's -i/-m/-M).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import READ_FN, WRITE_FN, CtasError, check, load

# bits per sample (the ct tool's -i) -> numpy type; 0 = float32
SAMPLE_TYPES = {0: np.float32, 8: np.uint8, -8: np.int8, 16: np.uint16, -16: np.int16,
                32: np.uint32, -32: np.int32, 64: np.uint64, -64: np.int64}


def sample_dtype(bpp: int):
    if bpp not in SAMPLE_TYPES:
        raise CtasError(-1, "bits per sample must be 0, +-8, +-16, +-32 or +-64")
    return np.dtype(SAMPLE_TYPES[bpp])


def quantize_dev(src, bpp: int, mincon: float = 0.0, maxcon: float = 0.0, out=None, stream=None):
    """limit<T> on the device: float32 CUDA tensor (n_images, ...) -> integer
    samples of bpp bits (a torch tensor of the matching type)."""
    import torch
    tmap = {8: torch.uint8, -8: torch.int8, 16: torch.uint16, -16: torch.int16,
            32: torch.uint32, -32: torch.int32, 64: torch.uint64, -64: torch.int64}
    if bpp not in tmap:
        raise CtasError(-1, "bits per sample must be one of +-8, +-16, +-32, +-64")
    if not (src.is_cuda and src.dtype == torch.float32 and src.is_contiguous() and src.dim() >= 1):
        raise CtasError(-1, "src must be a contiguous float32 CUDA tensor")
    if out is None:
        out = torch.empty(src.shape, dtype=tmap[bpp], device=src.device)
    n = int(src.shape[0])
    pixels = int(src.numel() // max(1, n))
    st = torch.cuda.current_stream().cuda_stream if stream is None else int(stream)
    check(load().ctas_vol_quantize_dev(C.c_void_p(src.data_ptr()), n, pixels, int(bpp),
                                       float(mincon), float(maxcon), C.c_void_p(out.data_ptr()),
                                       C.c_void_p(st)))
    return out


def reconstruct_volume(rec, n_slices: int, center: float, read, write, bpp: int = 0,
                       mincon: float = 0.0, maxcon: float = 0.0) -> None:
    """Stream n_slices sinograms through ``rec`` (a ``ct.CTrec``).

    ``read(first, count, sinos)`` fills the float32 array ``sinos``
    (count, N, W); ``write(first, count, slices)`` receives (count, rows, cols)
    samples of ``bpp`` (valid during the call only).  Both are called from
    library threads in slice order.  An exception in a callback ends the call
    and is re-raised here."""
    dt = sample_dtype(bpp)
    N, W = rec.ish
    rows, cols = rec.osh
    errors = []

    def _rd(_user, first, count, ptr):
        try:
            buf = (C.c_float * (count * N * W)).from_address(ptr)
            read(first, count, np.frombuffer(buf, np.float32).reshape(count, N, W))
            return 0
        except BaseException as e:  # reported after the call
            errors.append(e)
            return -1

    def _wr(_user, first, count, ptr):
        try:
            nbytes = count * rows * cols * dt.itemsize
            buf = (C.c_char * nbytes).from_address(ptr)
            write(first, count, np.frombuffer(buf, dt).reshape(count, rows, cols))
            return 0
        except BaseException as e:
            errors.append(e)
            return -1

    rd, wr = READ_FN(_rd), WRITE_FN(_wr)
    rc = load().ctas_fbp_reconstruct_volume(rec._h, int(n_slices), float(center), int(bpp),
                                            float(mincon), float(maxcon), rd, wr, None)
    if errors:
        raise errors[0]
    check(rc)


def reconstruct_arrays(rec, sinos: np.ndarray, center: float = 0.0, bpp: int = 0,
                       mincon: float = 0.0, maxcon: float = 0.0,
                       out: np.ndarray | None = None) -> np.ndarray:
    """The volume call over in-memory arrays: sinos (S, N, W) float32 ->
    slices (S, rows, cols) of bpp samples."""
    sinos = np.ascontiguousarray(sinos, np.float32)
    S = sinos.shape[0]
    if tuple(sinos.shape[1:]) != tuple(rec.ish):
        raise CtasError(-2, f"sinograms of shape {sinos.shape[1:]} for a {rec.ish} reconstruction")
    if out is None:
        out = np.empty((S,) + tuple(rec.osh), sample_dtype(bpp))

    def read(first, count, buf):
        np.copyto(buf, sinos[first:first + count])

    def write(first, count, buf):
        np.copyto(out[first:first + count], buf)

    reconstruct_volume(rec, S, center, read, write, bpp, mincon, maxcon)
    return out


def reconstruct_raw(rec, in_path: str, n_slices: int, out_path: str, center: float = 0.0,
                    bpp: int = 0, mincon: float = 0.0, maxcon: float = 0.0, *,
                    in_offset: int = 0, out_offset: int = 0, io_threads: int = 0) -> None:
    """Raw contiguous volumes: float32 (n_slices, N, W) at in_offset of
    in_path -> bpp samples (n_slices, rows, cols) at out_offset of out_path
    (created if absent, never truncated)."""
    check(load().ctas_vol_raw_reconstruct(rec._h, os.fsencode(in_path), int(in_offset),
                                          int(n_slices), os.fsencode(out_path), int(out_offset),
                                          float(center), int(bpp), float(mincon), float(maxcon),
                                          int(io_threads)))
