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
        L.icon_ws_conv3x3_wait_test.argtypes = [V, I, I, I, I, V, I, V, ctypes.c_uint, V]
        L.icon_ws_conv3x3_wait_test.restype = ctypes.c_int
        F, D, Z = ctypes.c_float, ctypes.c_double, ctypes.c_size_t
        L.icon_ws_create.argtypes = [P, I, ctypes.POINTER(P)]
        L.icon_ws_destroy.argtypes = [P]
        L.icon_ws_param_count.argtypes = []
        L.icon_ws_param_count.restype = Z
        L.icon_ws_init.argtypes = [P, ctypes.c_ulonglong]
        L.icon_ws_set_params.argtypes = [P, V, Z, F]
        L.icon_ws_get_params.argtypes = [P, V, Z, ctypes.POINTER(F)]
        L.icon_ws_set_gain.argtypes = [P, F]
        L.icon_ws_predict.argtypes = [P, V, V, I, V]
        L.icon_ws_backprop.argtypes = [P, V, V, I, ctypes.POINTER(D), V]
        L.icon_ws_get_grads.argtypes = [P, V, Z]
        L.icon_ws_update.argtypes = [P, F, V]
        L.icon_ws_train_step.argtypes = [P, V, V, I, F, ctypes.POINTER(D), V]
        L.icon_ws_load.argtypes = [P, ctypes.c_char_p]
        L.icon_plan_set_warm_start.argtypes = [P, P, V]
        L.icon_plan_warm_counts.argtypes = [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
        for name in ("icon_ws_create", "icon_ws_destroy", "icon_ws_init", "icon_ws_set_params", "icon_ws_get_params",
                     "icon_ws_set_gain", "icon_ws_predict", "icon_ws_backprop", "icon_ws_get_grads", "icon_ws_update",
                     "icon_ws_train_step", "icon_ws_load", "icon_plan_set_warm_start", "icon_plan_warm_counts"):
            getattr(L, name).restype = ctypes.c_int
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


def conv3x3_wait_test(in0, w, wait_us):
    """icon_ws_conv3x3_wait_test: a convolution whose first pipeline stage
    can never complete, so its bounded wait runs out after wait_us
    microseconds; returns the (skipped) output tensor."""
    import torch
    n, H, W, c0 = in0.shape
    N = w.shape[1]
    out0 = torch.zeros((n, H, W, N), dtype=torch.bfloat16, device=in0.device)
    _check(lib().icon_ws_conv3x3_wait_test(_ptr(in0), c0, n, H, W, _ptr(w), N, _ptr(out0), int(wait_us), _stream()))
    return out0


def param_count() -> int:
    return int(lib().icon_ws_param_count())


class Network:
    """The warm-start U-Net for the geometry of an IconPlan.

    Slices use the plan's layout: Ahwb (S, N0, N1) complex64 as returned by
    IconPlan.prepare_rhs, m (S, N0, N1) float32 as IconPlan.solve takes and
    returns.  predict() gives the start to pass as IconPlan.solve(m0=...)."""

    def __init__(self, plan, capacity=None):
        import torch
        self.plan = plan
        self.capacity = int(capacity or plan.capacity)
        h = ctypes.c_void_p()
        self._destroy = lib().icon_ws_destroy     # held so that __del__ works at interpreter exit
        with torch.cuda.device(plan.device):
            _check(lib().icon_ws_create(plan._h, self.capacity, ctypes.byref(h)))
        self._h = h
        self.n = param_count()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._destroy(h)
            self._h = None

    __del__ = close

    def init(self, seed=0):
        _check(lib().icon_ws_init(self._h, ctypes.c_ulonglong(int(seed))))

    def set_params(self, params, gain=1.0):
        import numpy as np
        p = np.ascontiguousarray(np.asarray(params, np.float32))
        if p.size != self.n:
            raise IconError(f"expected {self.n} parameters, got {p.size}")
        _check(lib().icon_ws_set_params(self._h, p.ctypes.data_as(ctypes.c_void_p), self.n, float(gain)))

    def get_params(self):
        import numpy as np
        p = np.zeros(self.n, np.float32)
        g = ctypes.c_float(0)
        _check(lib().icon_ws_get_params(self._h, p.ctypes.data_as(ctypes.c_void_p), self.n, ctypes.byref(g)))
        return p, float(g.value)

    def set_gain(self, gain):
        _check(lib().icon_ws_set_gain(self._h, float(gain)))

    def grads(self):
        import numpy as np
        p = np.zeros(self.n, np.float32)
        _check(lib().icon_ws_get_grads(self._h, p.ctypes.data_as(ctypes.c_void_p), self.n))
        return p

    def _in(self, Ahwb, m=None):
        import torch
        P = self.plan
        if Ahwb.dtype != torch.complex64 or not Ahwb.is_contiguous() or Ahwb.shape[1:] != (P.N0, P.N1):
            raise IconError("Ahwb must be a contiguous (S, N0, N1) complex64 tensor")
        if m is not None and (m.dtype != torch.float32 or not m.is_contiguous() or m.shape != Ahwb.shape):
            raise IconError("target must be a contiguous (S, N0, N1) float32 tensor")
        return Ahwb.shape[0]

    def predict(self, Ahwb, out=None):
        import torch
        S = self._in(Ahwb)
        if out is None:
            out = torch.empty((S, self.plan.N0, self.plan.N1), dtype=torch.float32, device=Ahwb.device)
        _check(lib().icon_ws_predict(self._h, _ptr(Ahwb), _ptr(out), S, _stream()))
        return out

    def backprop(self, Ahwb, target):
        S = self._in(Ahwb, target)
        loss = ctypes.c_double(0)
        _check(lib().icon_ws_backprop(self._h, _ptr(Ahwb), _ptr(target), S, ctypes.byref(loss), _stream()))
        return float(loss.value)

    def update(self, lr):
        _check(lib().icon_ws_update(self._h, float(lr), _stream()))

    def load(self, path):
        """Parameters and gain from a weights file written by save_raw."""
        _check(lib().icon_ws_load(self._h, str(path).encode()))

    def train_step(self, Ahwb, target, lr):
        S = self._in(Ahwb, target)
        loss = ctypes.c_double(0)
        _check(lib().icon_ws_train_step(self._h, _ptr(Ahwb), _ptr(target), S, float(lr), ctypes.byref(loss),
                                        _stream()))
        return float(loss.value)


WEIGHTS_DIR = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                         "weights")


def load_weights(path=None, nx=1024, thickness=300):
    """(params, gain, meta) of a trained network file (train_warmstart's
    output); by default the one shipped for nx x thickness."""
    import json
    import os
    import numpy as np
    path = path or os.path.join(WEIGHTS_DIR, f"warmstart_{nx}x{thickness}.npz")
    z = np.load(path)
    return z["params"].astype(np.float32), float(z["gain"]), json.loads(str(z["meta"]))


def save_raw(path, params, gain):
    """The weights file icon_ws_load reads (icon-gpu --warm-start): the 8
    bytes ICONWSB1, the parameter count (uint64), the gain (float32), then
    the FP32 parameters, little-endian."""
    import struct
    import numpy as np
    p = np.ascontiguousarray(np.asarray(params, "<f4"))
    with open(path, "wb") as f:
        f.write(b"ICONWSB1")
        f.write(struct.pack("<Qf", p.size, float(gain)))
        f.write(p.tobytes())


def set_warm_start(plan, net, tol, check_every=10, max_dist=2.0):
    """Warm start of the plan's reconstruct calls (icon_plan_set_warm_start);
    net None turns it off."""
    from .icon import WarmCfg
    if net is None:
        _check(lib().icon_plan_set_warm_start(plan._h, None, None))
        return
    wc = WarmCfg(float(tol), int(check_every), float(max_dist))
    _check(lib().icon_plan_set_warm_start(plan._h, net._h, ctypes.byref(wc)))


def warm_counts(plan):
    """(accepted, redone from zero) slices of the plan's warm-started reconstruct calls."""
    a, r = ctypes.c_longlong(0), ctypes.c_longlong(0)
    _check(lib().icon_plan_warm_counts(plan._h, ctypes.byref(a), ctypes.byref(r)))
    return int(a.value), int(r.value)


if __name__ == "__main__":
    # python -m feilab_b200.warmstart export WEIGHTS.npz OUT.bin
    import sys
    if len(sys.argv) == 4 and sys.argv[1] == "export":
        prm, g, _ = load_weights(sys.argv[2])
        save_raw(sys.argv[3], prm, g)
    else:
        print("usage: python -m feilab_b200.warmstart export WEIGHTS.npz OUT.bin")
        sys.exit(2)
