"""ctypes binding of ``libctas_fbp.so`` (the C ABI declared in include/*.h).

The library is loaded from this package directory.  There is no fallback: if
the library is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libctas_fbp.so")

OK = 0
E_ARG, E_SHAPE, E_CENTER, E_FILTER, E_DATA = -1, -2, -3, -4, -5
E_STATE, E_CUDA, E_NOMEM, E_UNSUPPORTED, E_NODEVICE, E_TIMEOUT = -6, -7, -8, -9, -10, -11
E_IO = -12

INTERP_TRUNC, INTERP_LINEAR = 0, 1
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
FLAG_NO_WRITEBACK = 0x1
FLAG_SHIPPED_INDEX = 0x2
FLAG_CHECKED = 0x100
FLAG_TEST_TIMEOUT = 0x200


class Opts(C.Structure):
    """ctas_fbp_opts"""
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("interp", C.c_int32),
        ("pad", C.c_int64),
        ("store", C.c_int32),
        ("device", C.c_int32),
        ("angles", C.POINTER(C.c_double)),
        ("out_rows", C.c_int64),
        ("out_cols", C.c_int64),
        ("out_pixel", C.c_double),
        ("out_shift_row", C.c_double),
        ("out_shift_col", C.c_double),
        ("flags", C.c_uint32),
        ("chunk_slices", C.c_int32),
        ("tile", C.c_int32),
        ("ring_box", C.c_int32),
    ]


class Job(C.Structure):
    """ctas_fbp_job"""
    _fields_ = [
        ("n_angles", C.c_int64),
        ("width", C.c_int64),
        ("center", C.c_float),
        ("sino_dev", C.c_void_p),
        ("slice_dev", C.c_void_p),
    ]


# name -> (restype, argtypes); every symbol declared in include/ctas_fbp.h
_P = C.c_void_p
_F = C.POINTER(C.c_float)
# include/ctas_volume.h callbacks
READ_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p)
WRITE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p)

SIGNATURES = {
    "ctas_fbp_last_error": (C.c_char_p, []),
    "ctas_fbp_version": (C.c_char_p, []),
    "ctas_filter_from_name": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "ctas_filter_name": (C.c_char_p, [C.c_int32]),
    "ctas_filter_check": (C.c_int, [C.c_int32, C.c_float]),
    "ctas_filter_parse": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), _F]),
    "ctas_filter_fill": (C.c_int, [C.c_int32, C.c_float, C.c_int64, _P]),
    "ctas_contrast_from_name": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "ctas_contrast_name": (C.c_char_p, [C.c_int32]),
    "ctas_fbp_padded_width": (C.c_int64, [C.c_int64]),
    "ctas_fbp_arc": (C.c_float, [C.c_float, C.c_int64]),
    "ctas_fbp_angle": (C.c_float, [C.c_float, C.c_int64]),
    "ctas_fbp_angle_table": (C.c_int, [C.c_float, C.c_int64, _P]),
    "ctas_fbp_window": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_int64, _P]),
    "ctas_fbp_rec_cof": (C.c_float, [C.c_float, C.c_float]),
    "ctas_fbp_create": (C.c_int, [C.POINTER(_P), C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                  C.c_float, C.c_float, C.POINTER(Opts)]),
    "ctas_fbp_clone": (C.c_int, [_P, C.POINTER(_P)]),
    "ctas_fbp_destroy": (C.c_int, [_P]),
    "ctas_fbp_set_physics": (C.c_int, [_P, C.c_float, C.c_float]),
    "ctas_fbp_rec_shape": (C.c_int, [_P, C.c_float, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "ctas_fbp_out_shape": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "ctas_fbp_sino_shape": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "ctas_fbp_sino": (C.c_int, [_P, _P]),
    "ctas_fbp_repeat": (C.c_int, [_P, _P, C.c_float]),
    "ctas_fbp_reconstruct": (C.c_int, [_P, _P, _P, C.c_float]),
    "ctas_fbp_sino_dev": (C.c_int, [_P, _P, _P, _P]),
    "ctas_fbp_repeat_dev": (C.c_int, [_P, _P, C.c_float, _P]),
    "ctas_fbp_repeat_multi_dev": (C.c_int, [_P, _P, C.c_int64, _P, _P]),
    "ctas_fbp_reconstruct_dev": (C.c_int, [_P, _P, _P, C.c_float, _P]),
    "ctas_fbp_synchronize": (C.c_int, [_P]),
    "ctas_fbp_reconstruct_stack": (C.c_int, [_P, _P, _P, C.c_int64, C.c_float]),
    "ctas_fbp_reconstruct_stack_dev": (C.c_int, [_P, _P, _P, C.c_int64, C.c_float, _P]),
    "ctas_fbp_last_kernel": (C.c_int, [_P]),
    "ctas_fbp_kernel_launches": (C.c_int64, [_P]),
    "ctas_fbp_last_tile": (C.c_int, [_P]),
    "ctas_fbp_tile_count": (C.c_int, []),
    "ctas_fbp_tile_shape": (C.c_int, [C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32)]),
    "ctas_fbp_batch_create": (C.c_int, [C.POINTER(_P), C.POINTER(Job), C.c_int64, C.c_int32,
                                        C.c_int32, C.c_float, C.c_float, C.c_float, C.c_float,
                                        C.POINTER(Opts)]),
    "ctas_fbp_batch_run": (C.c_int, [_P, _P]),
    "ctas_fbp_batch_run_loop": (C.c_int, [_P, _P]),
    "ctas_fbp_batch_synchronize": (C.c_int, [_P]),
    "ctas_fbp_batch_tile": (C.c_int, [_P]),
    "ctas_fbp_batch_destroy": (C.c_int, [_P]),
    "ctas_fbp_reconstruct_dev_noalloc": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int32,
                                                   C.c_int32, C.c_float, C.c_float, C.c_int64,
                                                   C.c_float, C.c_float, C.c_float, _P]),
    "ctas_fbp_set_profiling": (C.c_int, [_P, C.c_int]),
    "ctas_fbp_profile_read": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    # include/ctas_axis.h
    "ctas_ag_create": (C.c_int, [C.POINTER(_P), _P, C.c_int64, C.c_int64, C.c_float, C.c_int32]),
    "ctas_ag_create_flags": (C.c_int, [C.POINTER(_P), _P, C.c_int64, C.c_int64, C.c_float,
                                       C.c_int32, C.c_uint32]),
    "ctas_ag_apply": (C.c_int, [_P, _P, C.c_int64, _P]),
    "ctas_ag_sigma": (C.c_int, [_P, _F, C.POINTER(C.c_int32)]),
    "ctas_ag_destroy": (C.c_int, [_P]),
    "ctas_raxis": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_float, C.c_float, C.c_int32, C.c_int32,
                             _F, C.POINTER(C.c_int64)]),
    "ctas_raxis_pair": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_float, C.c_int32, _F]),
    # include/ctas_ts.h
    "ctas_ts_create": (C.c_int, [C.POINTER(_P), C.c_int64, C.c_int64, C.c_int32, C.c_float,
                                 C.c_int32, C.c_int32]),
    "ctas_ts_destroy": (C.c_int, [_P]),
    "ctas_ts_add": (C.c_int, [_P, _P, _P, C.c_float, C.c_float, C.c_int32, C.c_uint32]),
    "ctas_ts_add_dev": (C.c_int, [_P, _P, _P, C.c_float, C.c_float, C.c_int32, C.c_uint32, _P]),
    "ctas_ts_add_batch_dev": (C.c_int, [_P, _P, _P, C.c_int64, _P, C.c_float, C.c_int32,
                                        C.c_uint32, _P]),
    # include/ctas_learned.h
    "ctas_unet_create": (C.c_int, [C.POINTER(_P), C.c_uint64, C.c_int32]),
    "ctas_unet_destroy": (C.c_int, [_P]),
    "ctas_unet_set_scale": (C.c_int, [_P, C.c_float]),
    "ctas_unet_forward_dev": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, C.c_int64, _P]),
    "ctas_unet_train_step_dev": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_float,
                                           C.POINTER(C.c_double), _P]),
    "ctas_unet_param_count": (C.c_int64, [_P]),
    "ctas_unet_get_params": (C.c_int, [_P, _P]),
    "ctas_unet_set_params": (C.c_int, [_P, _P]),
    "ctas_unet_macs_per_pixel": (C.c_double, []),
    "ctas_nn_conv3x3_dev": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32,
                                      C.c_int32, C.c_int32, _P, C.c_int32, C.c_int32, C.c_int64,
                                      C.c_int64, C.c_int64, C.c_int32, _P]),
    "ctas_nn_conv3x3_wgrad_dev": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32,
                                            C.c_int32, C.c_int32, _P, C.c_int64, C.c_int64,
                                            C.c_int64, _P]),
    "ctas_nn_flip_weights_dev": (C.c_int, [_P, C.c_int32, C.c_int32, _P, _P]),
    "ctas_nn_test_timeout": (C.c_int, [C.c_int32]),
    # include/ctas_volume.h
    "ctas_vol_sample_bytes": (C.c_int32, [C.c_int32]),
    "ctas_vol_quantize_dev": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int32, C.c_float, C.c_float,
                                        _P, _P]),
    "ctas_fbp_reconstruct_volume": (C.c_int, [_P, C.c_int64, C.c_float, C.c_int32, C.c_float,
                                              C.c_float, READ_FN, WRITE_FN, _P]),
    "ctas_vol_raw_reconstruct": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, C.c_char_p,
                                           C.c_int64, C.c_float, C.c_int32, C.c_float, C.c_float,
                                           C.c_int32]),
    # include/ctas_probe.h
    "ctas_probe_smem_gather": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ctas_probe_l2_read": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ctas_probe_bounded_wait": (C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_double)]),
    # include/ctas_phantom.h
    "ctas_phantom_sinogram_dev": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P,
                                            C.c_double, _P, _P]),
    "ctas_phantom_project_image_dev": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, _P,
                                                 C.c_double, C.c_double, C.c_double, _P, _P]),
}

_lib = None
_lock = threading.Lock()


class CtasError(RuntimeError):
    """Raised for a non-zero status; mirrors ctas' CtasErr
    (src/common/common.world.h:155-176)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


def load():
    """Load the native library (fails loudly if it is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"{LIB_PATH} is missing: build it with "
                              "`python ctas_b200/build.py` (there is no fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != OK:
        msg = load().ctas_fbp_last_error().decode(errors="replace")
        raise CtasError(rc, msg)
    return rc
