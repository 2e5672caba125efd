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


def _mask_lib():
    L = lib()
    if not getattr(L, "_mask_ready", False):
        P, I, V, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_float
        L.icon_mask_radius.argtypes = [I, V, I, I, V, V, I, ctypes.POINTER(F), ctypes.POINTER(F), ctypes.POINTER(I)]
        L.icon_mask_create.argtypes = [I, V, I, F, F, I, I, I, ctypes.POINTER(P)]
        L.icon_mask_destroy.argtypes = [P]
        L.icon_mask_filter.argtypes = [P, V]
        L.icon_mask_apply.argtypes = [P, V, I, I, I, V, V]
        L.icon_volume_crop.argtypes = [V, I, I, I, I, V, V]
        for n in ("icon_mask_radius", "icon_mask_create", "icon_mask_destroy", "icon_mask_filter", "icon_mask_apply",
                  "icon_volume_crop"):
            getattr(L, n).restype = ctypes.c_int
        L._mask_ready = True
    return L


def mask_radius(n, tilts, radius=None, crossv=None, fullrec=None):
    """(rate of the FRC-0.5 radius, rate of the FRC-0.3 radius, explicit?)
    as ICONMask3 derives them; radius None reads the FRC curves."""
    t = np.ascontiguousarray(np.asarray(tilts, np.float32))
    cv = np.ascontiguousarray(np.asarray(crossv, np.float32)) if crossv is not None else None
    fr = np.ascontiguousarray(np.asarray(fullrec, np.float32)) if fullrec is not None else None
    r05, r03, ex = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
    _check(_mask_lib().icon_mask_radius(int(n), t.ctypes.data_as(ctypes.c_void_p), t.size,
                                        -1 if radius is None else int(radius),
                                        cv.ctypes.data_as(ctypes.c_void_p) if cv is not None else None,
                                        fr.ctypes.data_as(ctypes.c_void_p) if fr is not None else None,
                                        min(cv.size, fr.size) if cv is not None and fr is not None else 0,
                                        ctypes.byref(r05), ctypes.byref(r03), ctypes.byref(ex)))
    return float(r05.value), float(r03.value), bool(ex.value)


class Mask:
    """ICONMask3's cross-validation mask for n x n slices on the GPU."""

    def __init__(self, n, tilts, rate05, rate03, explicit, gauss_width=None, capacity=16):
        t = np.ascontiguousarray(np.asarray(tilts, np.float32))
        h = ctypes.c_void_p()
        self._destroy = _mask_lib().icon_mask_destroy     # held so that __del__ works at interpreter exit
        _check(_mask_lib().icon_mask_create(int(n), t.ctypes.data_as(ctypes.c_void_p), t.size, float(rate05),
                                            float(rate03), int(explicit), int(gauss_width or 0), int(capacity),
                                            ctypes.byref(h)))
        self._h, self.n, self.capacity = h, int(n), int(capacity)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def filter(self):
        f = np.zeros((self.n, self.n // 2 + 1), np.float32)
        _check(_mask_lib().icon_mask_filter(self._h, f.ctypes.data_as(ctypes.c_void_p)))
        return f

    def apply(self, slices, ystart, thickness):
        """slices (S, n, n) float32 CUDA tensor -> (S, thickness, n)."""
        import torch
        S = slices.shape[0]
        out = torch.empty((S, thickness, self.n), dtype=torch.float32, device=slices.device)
        _check(_mask_lib().icon_mask_apply(self._h, ctypes.c_void_p(slices.data_ptr()), S, int(ystart),
                                           int(thickness), ctypes.c_void_p(out.data_ptr()), _stream()))
        return out


def frc(a, b, smooth_overlap=10):
    """FRC of two (ny, nx) images as the reference's cross validation
    computes it (calFRC_nonsqure, then frcSmooth); nx/2 values."""
    L = lib()
    if not getattr(L, "_frc_ready", False):
        L.icon_frc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_void_p]
        L.icon_frc.restype = ctypes.c_int
        L._frc_ready = True
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    b = np.ascontiguousarray(np.asarray(b, np.float32))
    if a.shape != b.shape or a.ndim != 2:
        raise IconError("frc: two images of the same (ny, nx) shape are needed")
    ny, nx = a.shape
    out = np.zeros(nx // 2, np.float32)
    _check(L.icon_frc(a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p), nx, ny,
                      int(smooth_overlap), out.ctypes.data_as(ctypes.c_void_p)))
    return out


def loo_sweep(rows, thickness, tilts, iters=(0, 10, 0), data_type=1, threshold=0.03, capacity=64, tol=0.0,
              device=0, operator="nufft"):
    """Leave-one-out cross validation over every tilt: rows (S, nz, nx)
    float32 (host); operator "nufft" or "toeplitz" (the iterations' normal
    operator).  Returns (frc (nz, nx/2), reprojections (nz, S, nx),
    iterations per omitted tilt (nz,))."""
    from .icon import SolveCfg
    L = lib()
    if not getattr(L, "_loo_ready", False):
        V, I = ctypes.c_void_p, ctypes.c_int
        L.icon_loo_sweep.argtypes = [V, I, I, I, V, ctypes.POINTER(SolveCfg), I, I, ctypes.c_double, I, V, V, V, I]
        L.icon_loo_sweep.restype = ctypes.c_int
        L._loo_ready = True
    r = np.ascontiguousarray(np.asarray(rows, np.float32))
    S, nz, nx = r.shape
    t = np.ascontiguousarray(np.asarray(tilts, np.float32))
    a, b, c = iters
    cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
    f = np.zeros((nz, nx // 2), np.float32)
    rp = np.zeros((nz, S, nx), np.float32)
    it = np.zeros(nz, np.int32)
    _check(L.icon_loo_sweep(r.ctypes.data_as(ctypes.c_void_p), nx, int(thickness), nz, t.ctypes.data_as(ctypes.c_void_p),
                            ctypes.byref(cfg), S, int(capacity), float(tol), int(device),
                            f.ctypes.data_as(ctypes.c_void_p), rp.ctypes.data_as(ctypes.c_void_p),
                            it.ctypes.data_as(ctypes.c_void_p), {"nufft": 0, "toeplitz": 1}[operator]))
    return f, rp, it
