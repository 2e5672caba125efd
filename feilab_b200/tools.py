"""Python binding of include/icon_tools.h: the GPU versions of the
reference's companion tools around the ICON solve."""
from __future__ import annotations

import ctypes

import numpy as np

from .icon import IconError, _check, _stream, lib as _icon_lib

_ready = False


def lib():
    global _ready
    L = _icon_lib()
    if not _ready:
        P, I, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
        L.icon_preprocess.argtypes = [V, V, I, I, I, V, I, V]
        L.icon_preprocess.restype = ctypes.c_int
        L.icon_preprocess_host.argtypes = [V, V, I, I, I, V, I]
        L.icon_preprocess_host.restype = ctypes.c_int
        _ready = True
    return L


def preprocess(stack, tilts=None, thickness=None, out=None):
    """ICONPreProcess on a (nz, ny, nx) float32 CUDA tensor: mode subtraction,
    and with tilts and thickness the variance normalisation.  Returns out
    (a new tensor, or `out`, which may be `stack` itself)."""
    import torch
    if stack.dtype != torch.float32 or not stack.is_cuda or not stack.is_contiguous() or stack.dim() != 3:
        raise IconError("stack must be a contiguous (nz, ny, nx) float32 CUDA tensor")
    nz, ny, nx = stack.shape
    if out is None:
        out = torch.empty_like(stack)
    t = None
    if tilts is not None and thickness:
        t = np.ascontiguousarray(np.asarray(tilts, np.float32))
        if t.size < nz:
            raise IconError("one tilt angle per projection is needed")
    _check(lib().icon_preprocess(ctypes.c_void_p(stack.data_ptr()), ctypes.c_void_p(out.data_ptr()), nx, ny, nz,
                                 t.ctypes.data_as(ctypes.c_void_p) if t is not None else None,
                                 int(thickness) if t is not None else 0, _stream()))
    return out
