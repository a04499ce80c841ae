"""The learned sparse-angle stage (extension; no counterpart in the reference).

Python face of include/ctas_learned.h: ``UNet`` (4-level U-Net, BF16 with FP32
accumulation, hand-written forward / backward / Adam kernels) and the layer
entry points it is built from.  Tensors are torch CUDA tensors; images FP32
(B, H, W) with H % 64 == 0 and W % 128 == 0; layer activations BF16 NHWC.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import CtasError, check, load


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(stream)


def _img(t, what):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
            and t.is_contiguous() and t.dim() == 3):
        raise CtasError(-1, f"{what} must be a contiguous float32 CUDA tensor (B, H, W)")
    return t


class UNet:
    """``UNet(seed, scale)``: He-initialised network (zero head: starts as the
    identity).  ``forward(x)`` returns x + net(x * scale) / scale;
    ``train_step(x, target, lr)`` runs one Adam step on the mean squared error
    (scaled units) and returns that error before the step."""

    def __init__(self, seed: int = 0, scale: float = 1.0, *, device: int = -1):
        self._h = None
        h = C.c_void_p()
        check(load().ctas_unet_create(C.byref(h), int(seed), int(device)))
        self._h = h
        self.set_scale(scale)

    def set_scale(self, scale: float):
        check(load().ctas_unet_set_scale(self._h, float(scale)))
        self.scale = float(scale)

    def forward(self, x, out=None, stream=None):
        import torch
        _img(x, "x")
        if out is None:
            out = torch.empty_like(x)
        B, H, W = x.shape
        check(load().ctas_unet_forward_dev(self._h, _ptr(x), _ptr(out), B, H, W, _stream(stream)))
        return out

    def train_step(self, x, target, lr: float = 1e-3, stream=None) -> float:
        _img(x, "x")
        _img(target, "target")
        if tuple(x.shape) != tuple(target.shape):
            raise CtasError(-2, "x and target shapes differ")
        B, H, W = x.shape
        loss = C.c_double()
        check(load().ctas_unet_train_step_dev(self._h, _ptr(x), _ptr(target), B, H, W, float(lr),
                                              C.byref(loss), _stream(stream)))
        return loss.value

    @property
    def param_count(self) -> int:
        return int(load().ctas_unet_param_count(self._h))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.param_count, np.float32)
        check(load().ctas_unet_get_params(self._h, p.ctypes.data_as(C.c_void_p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.param_count:
            raise CtasError(-1, "parameter vector of the wrong length")
        check(load().ctas_unet_set_params(self._h, p.ctypes.data_as(C.c_void_p)))

    @staticmethod
    def macs_per_pixel() -> float:
        return float(load().ctas_unet_macs_per_pixel())

    def close(self):
        if self._h:
            load().ctas_unet_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# layer table of the network, in parameter order: (cin, cout)
LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128), (128, 256), (256, 256),
          (384, 128), (128, 128), (192, 64), (64, 64), (96, 32), (32, 32)]
HEAD_C = 32


def split_params(p: np.ndarray):
    """Parameter vector -> list of (w[cout][9][cin], bias[cout]) and the head."""
    out, o = [], 0
    for cin, cout in LAYERS:
        w = p[o:o + cout * 9 * cin].reshape(cout, 9, cin)
        o += cout * 9 * cin
        b = p[o:o + cout]
        o += cout
        out.append((w, b))
    hw = p[o:o + HEAD_C]
    hb = p[o + HEAD_C]
    return out, hw, hb


# ------------------------------------------------------------------ layers
def conv3x3(x, w, bias=None, *, cin=None, x_co=0, y=None, y_co=0, cout=None, mask=None, m_co=0,
            relu=True, stream=None):
    """y[..., y_co:y_co+cout] = act(conv3x3(x[..., x_co:x_co+cin], w) + bias) on
    BF16 NHWC tensors (B, H, W, C); w BF16 (cout, 9, cin)."""
    import torch
    B, H, W, xc = x.shape
    cout = cout or w.shape[0]
    cin = cin or w.shape[2]
    if y is None:
        y = torch.empty((B, H, W, cout), dtype=torch.bfloat16, device=x.device)
    check(load().ctas_nn_conv3x3_dev(_ptr(x), xc, x_co, cin, _ptr(w), _ptr(bias), _ptr(y),
                                     y.shape[3], y_co, cout, _ptr(mask),
                                     mask.shape[3] if mask is not None else 0, m_co, B, H, W,
                                     1 if relu else 0, _stream(stream)))
    return y


def conv3x3_wgrad(x, dy, dw, *, cin=None, x_co=0, cout=None, dy_co=0, stream=None):
    """dw (FP32, (cout, 9, cin)) += weight gradient of conv3x3(x) for output
    gradient dy (BF16 NHWC)."""
    B, H, W, xc = x.shape
    cin = cin or dw.shape[2]
    cout = cout or dw.shape[0]
    check(load().ctas_nn_conv3x3_wgrad_dev(_ptr(x), xc, x_co, cin, _ptr(dy), dy.shape[3], dy_co,
                                           cout, _ptr(dw), B, H, W, _stream(stream)))
    return dw


def flip_weights(w, stream=None):
    """(cout, 9, cin) -> (cin, 9, cout) with the taps reversed: the weights of
    the data gradient."""
    import torch
    cout, _, cin = w.shape
    wt = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device=w.device)
    check(load().ctas_nn_flip_weights_dev(_ptr(w), cout, cin, _ptr(wt), _stream(stream)))
    return wt
