"""Python binding of include/icon_warmstart.h: the learned warm start.

The reference starts every ICON solve from m = 0 (IG/Iteration2.cu:33).  This
module binds the library's U-Net (BF16 on the sm_100a tensor cores) that
predicts a start from the slice's back-projection Re(A^H W b); the solve that
follows is the reference's algorithm unchanged.  Device arrays are torch
CUDA tensors; work is queued on torch's current stream.
"""
from __future__ import annotations

import ctypes

from .icon import IconError, _check, _stream, lib as _icon_lib

_ws_ready = False


def lib():
    global _ws_ready
    L = _icon_lib()
    if not _ws_ready:
        P, I, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
        L.icon_ws_conv3x3.argtypes = [V, I, V, I, I, I, I, V, V, I, I, V, I, I, V, I, V]
        L.icon_ws_conv3x3.restype = ctypes.c_int
        L.icon_ws_device_error.argtypes = [ctypes.POINTER(I)]
        L.icon_ws_device_error.restype = ctypes.c_int
        _ws_ready = True
    return L


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def device_error() -> int:
    """Reads and clears the device error flag of the tensor-core kernels."""
    v = ctypes.c_int(0)
    _check(lib().icon_ws_device_error(ctypes.byref(v)))
    return int(v.value)


def conv3x3(in0, w, bias=None, relu=False, in1=None, nsplit=None, out0=None, out1=None, acc0=False, acc1=False):
    """3x3 convolution (stride 1, zero padding 1) on the tensor cores.

    in0: [n, H, W, c0] bf16 (NHWC); in1: optional [n, H, W, c1] bf16, read as
    channels c0.. of one concatenated input; w: [9, N, c0 + c1] bf16 with
    tap = 3*dy + dx; bias: [N] float32 or None.  Returns out0 [n, H, W, nsplit]
    (and out1 [n, H, W, N - nsplit] when nsplit < N), bf16."""
    import torch
    n, H, W, c0 = in0.shape
    c1 = in1.shape[3] if in1 is not None else 0
    N = w.shape[1]
    if w.shape != (9, N, c0 + c1):
        raise IconError(f"conv3x3: weight shape {tuple(w.shape)} does not match inputs")
    for t in (in0, in1, w, out0, out1):
        if t is not None and (t.dtype != torch.bfloat16 or not t.is_contiguous()):
            raise IconError("conv3x3: activations and weights must be contiguous bf16")
    if bias is not None and (bias.dtype != torch.float32 or bias.numel() != N):
        raise IconError("conv3x3: bias must be float32 [N]")
    nsplit = N if nsplit is None else nsplit
    if out0 is None:
        out0 = torch.empty((n, H, W, nsplit), dtype=torch.bfloat16, device=in0.device)
    if nsplit < N and out1 is None:
        out1 = torch.empty((n, H, W, N - nsplit), dtype=torch.bfloat16, device=in0.device)
    _check(lib().icon_ws_conv3x3(_ptr(in0), c0, _ptr(in1), c1, n, H, W, _ptr(w), _ptr(bias), N, int(relu),
                                 _ptr(out0), nsplit, int(acc0), _ptr(out1), int(acc1), _stream()))
    return (out0, out1) if nsplit < N else out0
