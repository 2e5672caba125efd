"""Python binding of the C ABI in include/icon_b200.h (ctypes, torch tensors).

This mirrors the reference's per-slice routines of ICON-GPU v1.2.9
(nufft_gpu_v8.cu: cunfft_trafo_2d_R2C2, cunfft_trafo_2d2, cunfft_adjoint_2d2;
readSlicePart; Iteration3; reProject_NFFT2) as batched calls on a plan.  All
device arrays are torch CUDA tensors on the plan's device; work is queued on
torch's current stream.  Errors raise IconError with the library's message.

The library must have been built (python -m feilab_b200.build); there is no
fallback: importing on a machine without it raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libicon_b200.so")

_lib = None


class IconError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise IconError(f"native library {LIB_PATH} is missing; build it with `python -m feilab_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, I, F, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_void_p
        L.icon_plan_create.argtypes = [ctypes.POINTER(Geometry), ctypes.POINTER(P)]
        L.icon_plan_destroy.argtypes = [P]
        L.icon_plan_query.argtypes = [P, ctypes.POINTER(I)]
        L.icon_plan_geometry.argtypes = [P, V, V]
        L.icon_nufft_forward.argtypes = [P, V, V, I, V]
        L.icon_nufft_forward_complex.argtypes = [P, V, V, I, V]
        L.icon_nufft_adjoint.argtypes = [P, V, V, I, V]
        L.icon_rows_forward.argtypes = [P, V, V, I, V]
        L.icon_prepare_rhs.argtypes = [P, V, V, I, V]
        L.icon_solve.argtypes = [P, ctypes.POINTER(SolveCfg), V, V, I, I, V, V, V]
        L.icon_solve_warm.argtypes = [P, ctypes.POINTER(SolveCfg), V, V, I, ctypes.POINTER(WarmCfg), V,
                                      ctypes.POINTER(I), V]
        L.icon_solve_until.argtypes = [P, ctypes.POINTER(SolveCfg), V, V, I, I, ctypes.c_double, I,
                                       ctypes.POINTER(I), V, V]
        L.icon_reproject.argtypes = [P, V, F, V, I, V]
        L.icon_reconstruct_host.argtypes = [P, ctypes.POINTER(SolveCfg), V, V, V, I, V]
        L.icon_prepare_rhs_stack.argtypes = [P, V, I, I, I, V, I, V]
        L.icon_reconstruct_stack.argtypes = [P, ctypes.POINTER(SolveCfg), V, I, I, I, V, V, I, V]
        L.icon_reconstruct_stack_host.argtypes = [P, ctypes.POINTER(SolveCfg), V, I, I, I, I, I, BATCH_SINK, V, V]
        L.icon_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(V)]
        L.icon_host_free.argtypes = [V]
        L.icon_stack_upload.argtypes = [I, V, I, I, I, I, I, ctypes.POINTER(V), V]
        L.icon_device_free.argtypes = [I, V]
        L.icon_weights.argtypes = [I, I, V, V]
        L.icon_plan_set_group_weights.argtypes = [P, V, I]
        L.icon_plan_set_operator.argtypes = [P, I]
        L.icon_plan_set_stop.argtypes = [P, ctypes.c_double, I]
        L.icon_reproject_host.argtypes = [P, V, F, V, I, V]
        L.icon_batch_create.argtypes = [V, I, I, I, ctypes.c_char_p, I, ctypes.POINTER(V)]
        L.icon_batch_destroy.argtypes = [V]
        L.icon_batch_tuning.argtypes = [V, I, V]
        L.icon_batch_reconstruct_host.argtypes = [V, ctypes.POINTER(SolveCfg), V, V, I]
        L.icon_trace_enable.argtypes = [P, I]
        L.icon_trace_read.argtypes = [P, V, V, V]
        L.icon_launch_count.argtypes = [P]
        L.icon_launch_count.restype = ctypes.c_longlong
        L.icon_plan_device_error.argtypes = [P, ctypes.POINTER(I)]
        L.icon_last_error.restype = ctypes.c_char_p
        for name in ("icon_plan_create", "icon_plan_destroy", "icon_plan_query", "icon_plan_geometry",
                     "icon_nufft_forward", "icon_nufft_forward_complex", "icon_nufft_adjoint",
                     "icon_rows_forward", "icon_prepare_rhs", "icon_solve", "icon_solve_until", "icon_solve_warm", "icon_reproject",
                     "icon_reconstruct_host", "icon_trace_enable", "icon_trace_read", "icon_prepare_rhs_stack",
                     "icon_reconstruct_stack", "icon_reconstruct_stack_host", "icon_host_alloc", "icon_host_free",
                     "icon_stack_upload", "icon_device_free", "icon_weights", "icon_plan_set_group_weights",
                     "icon_plan_set_operator", "icon_plan_set_stop", "icon_reproject_host", "icon_batch_create",
                     "icon_batch_destroy", "icon_batch_tuning", "icon_batch_reconstruct_host",
                     "icon_plan_device_error"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


# icon_batch_sink: int (*)(void *ctx, int s0, int count, const float *h_slices, const float *h_reproj)
BATCH_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_void_p)
OUT_SLICES, OUT_REPROJECTION = 1, 2


class Geometry(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("thickness", ctypes.c_int), ("ntilt", ctypes.c_int),
                ("tilt_deg", ctypes.POINTER(ctypes.c_float)), ("capacity", ctypes.c_int), ("device", ctypes.c_int),
                ("window", ctypes.c_int)]


# NUFFT windows (ICON_WINDOW_*): the reference's Gaussian (half-width 6, 14
# taps) and the Kaiser-Bessel window of half-width 4 (8 taps).
WINDOWS = {"gauss6": 0, "kb4": 1}


class WarmCfg(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("check_every", ctypes.c_int), ("max_dist", ctypes.c_double)]


# Per-slice outcome of IconPlan.solve_warm (ICON_WARM_*).
WARM_OUTCOMES = {0: "accepted", 1: "not finite", 2: "not converged", 3: "too far from the cold INFR iterate"}


class SolveCfg(ctypes.Structure):
    _fields_ = [("infr_before", ctypes.c_int), ("icon", ctypes.c_int), ("infr_after", ctypes.c_int),
                ("data_type", ctypes.c_int), ("threshold", ctypes.c_float)]


def _check(rc):
    if rc != 0:
        msg = lib().icon_last_error().decode(errors="replace")
        raise IconError(f"icon status {rc}: {msg}")


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class IconPlan:
    """Plan for one tilt series: nx detector pixels, `thickness` (0 = nx)
    reconstruction rows, tilt angles as in the .tlt file, up to `capacity`
    slices per call; window "gauss6" (the reference's) or "kb4"."""

    def __init__(self, nx, thickness, tilts, capacity=8, device=None, window="gauss6"):
        import torch
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device)
        self.tilts = np.ascontiguousarray(np.asarray(tilts, np.float32))
        g = Geometry(int(nx), int(thickness), len(self.tilts),
                     self.tilts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(capacity), int(device),
                     WINDOWS[window])
        self.window = window
        h = ctypes.c_void_p()
        self._destroy = lib().icon_plan_destroy     # held so that __del__ works at interpreter exit
        _check(lib().icon_plan_create(ctypes.byref(g), ctypes.byref(h)))
        self._h = h
        d = (ctypes.c_int * 10)()
        _check(lib().icon_plan_query(h, d))
        self.N0, self.N1, self.n0, self.n1, self.M, self.nz, self.B, self.capacity, self.mib, self.omit_index = list(d)
        self.nx = self.N0

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._destroy(h)
            self._h = None

    __del__ = close

    def set_group_weights(self, w=None):
        """Per-group density weights (ngroups, M) float32 for slice groups
        0..ngroups-1 of later calls (B slices each); None restores the
        plan's own weights."""
        if w is None:
            _check(lib().icon_plan_set_group_weights(self._h, None, 0))
            return
        w = np.ascontiguousarray(np.asarray(w, np.float32).reshape(-1, self.M))
        _check(lib().icon_plan_set_group_weights(self._h, w.ctypes.data_as(ctypes.c_void_p), w.shape[0]))

    OPERATORS = {"nufft": 0, "toeplitz": 1}

    def set_operator(self, op):
        """Normal operator of the iterations: "nufft" (the reference's NUFFT
        pair, default) or "toeplitz" (A^H W A as a convolution with the exact
        kernel of the node set; see icon_plan_set_operator)."""
        _check(lib().icon_plan_set_operator(self._h, self.OPERATORS[op]))
        self.operator = op

    def set_stop(self, tol=0.0, check_every=10):
        """Tolerance stop of the reconstruct calls (icon_plan_set_stop): their
        ICON phase ends once every slice's relative step is within tol;
        tol = 0 runs the whole schedule."""
        _check(lib().icon_plan_set_stop(self._h, float(tol), int(check_every)))

    def geometry(self):
        xy = np.zeros((self.M, 2), np.float32)
        w = np.zeros(self.M, np.float32)
        _check(lib().icon_plan_geometry(self._h, xy.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p)))
        return xy, w

    def _dev(self, t, dtype):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.device == self.device and t.dtype == dtype and t.is_contiguous()):
            raise IconError(f"expected a contiguous {dtype} tensor on {self.device}")
        return t

    def nufft_forward(self, img):
        """img (S, N0, N1) float32 or complex64 -> nodes (S, M) complex64."""
        import torch
        S = img.shape[0]
        out = torch.empty((S, self.M), dtype=torch.complex64, device=self.device)
        if img.dtype == torch.complex64:
            _check(lib().icon_nufft_forward_complex(self._h, _ptr(self._dev(img, torch.complex64)), _ptr(out), S, _stream()))
        else:
            _check(lib().icon_nufft_forward(self._h, _ptr(self._dev(img, torch.float32)), _ptr(out), S, _stream()))
        return out

    def nufft_adjoint(self, f):
        """f (S, M) complex64 -> image (S, N0, N1) complex64."""
        import torch
        S = f.shape[0]
        out = torch.empty((S, self.N0, self.N1), dtype=torch.complex64, device=self.device)
        _check(lib().icon_nufft_adjoint(self._h, _ptr(self._dev(f, torch.complex64)), _ptr(out), S, _stream()))
        return out

    def rows_forward(self, rows):
        """rows (S, nz, nx) float32 -> b (S, M) complex64."""
        import torch
        S = rows.shape[0]
        out = torch.empty((S, self.M), dtype=torch.complex64, device=self.device)
        _check(lib().icon_rows_forward(self._h, _ptr(self._dev(rows, torch.float32)), _ptr(out), S, _stream()))
        return out

    def prepare_rhs(self, rows):
        """rows (S, nz, nx) float32 -> A^H W b (S, N0, N1) complex64."""
        import torch
        S = rows.shape[0]
        out = torch.empty((S, self.N0, self.N1), dtype=torch.complex64, device=self.device)
        _check(lib().icon_prepare_rhs(self._h, _ptr(self._dev(rows, torch.float32)), _ptr(out), S, _stream()))
        return out

    def solve(self, Ahwb, iters=(0, 10, 0), data_type=1, threshold=0.03, m0=None, history=False):
        """Iteration3 on S slices; returns m (S, N0, N1) float32 (and, with
        history=True, alpha and ||rhat||^2 per iteration as (iters, S))."""
        import torch
        S = Ahwb.shape[0]
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        if m0 is None:
            m = torch.empty((S, self.N0, self.N1), dtype=torch.float32, device=self.device)
            warm = 0
        else:
            m = self._dev(m0, torch.float32).clone()
            warm = 1
        n = a + b + c
        ha = np.zeros((max(n, 1), S), np.float64) if history else None
        hr = np.zeros((max(n, 1), S), np.float64) if history else None
        _check(lib().icon_solve(self._h, ctypes.byref(cfg), _ptr(self._dev(Ahwb, torch.complex64)), _ptr(m), S, warm,
                                ha.ctypes.data_as(ctypes.c_void_p) if history else None,
                                hr.ctypes.data_as(ctypes.c_void_p) if history else None, _stream()))
        if history:
            return m, ha[:n], hr[:n]
        return m

    def solve_until(self, Ahwb, tol=0.0, iters=(0, 10, 0), data_type=1, threshold=0.03, m0=None, check_every=10):
        """Iteration3 whose ICON phase ends once every slice's relative step
        ||m_new - m_old|| / ||m_new|| is at or below tol (checked every
        check_every ICON iterations).  Returns (m, iterations done, relative
        step per slice at the last check)."""
        import torch
        S = Ahwb.shape[0]
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        if m0 is None:
            m = torch.empty((S, self.N0, self.N1), dtype=torch.float32, device=self.device)
            warm = 0
        else:
            m = self._dev(m0, torch.float32).clone()
            warm = 1
        n = ctypes.c_int(0)
        step = np.zeros(S, np.float64)
        _check(lib().icon_solve_until(self._h, ctypes.byref(cfg), _ptr(self._dev(Ahwb, torch.complex64)), _ptr(m), S,
                                      warm, float(tol), int(check_every), ctypes.byref(n),
                                      step.ctypes.data_as(ctypes.c_void_p), _stream()))
        return m, int(n.value), step

    def solve_warm(self, Ahwb, m0, tol, iters=(0, 10, 0), data_type=1, threshold=0.03, check_every=10, max_dist=2.0):
        """Warm-started solve from m0 with the cold start as judge and
        fallback (icon_solve_warm): returns (m, per-slice outcome codes
        ICON_WARM_* as an int array, 0 = accepted, else redone from m = 0,
        iterations of the warm solve)."""
        import torch
        S = Ahwb.shape[0]
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        wc = WarmCfg(float(tol), int(check_every), float(max_dist))
        m = self._dev(m0, torch.float32).clone()
        redone = np.zeros(S, np.int32)
        n = ctypes.c_int(0)
        _check(lib().icon_solve_warm(self._h, ctypes.byref(cfg), _ptr(self._dev(Ahwb, torch.complex64)), _ptr(m), S,
                                     ctypes.byref(wc), redone.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n),
                                     _stream()))
        return m, redone, int(n.value)

    def reproject(self, m, tilt_deg=None):
        """m (S, N0, N1) float32 -> (S, nx) float32 reprojection at tilt_deg
        (.tlt value; default the smallest-|angle| tilt, as Lib_2D2 does)."""
        import torch
        S = m.shape[0]
        if tilt_deg is None:
            tilt_deg = float(self.tilts[self.omit_index])
        out = torch.empty((S, self.nx), dtype=torch.float32, device=self.device)
        _check(lib().icon_reproject(self._h, _ptr(self._dev(m, torch.float32)), ctypes.c_float(tilt_deg), _ptr(out), S, _stream()))
        return out

    def reconstruct_host(self, rows, iters=(0, 10, 0), data_type=1, threshold=0.03, reproject=False, out=None,
                         stream=None):
        """Host arrays in and out: rows (S, nz, nx) float32 -> m (S, N0, N1)
        (and the reprojection (S, nx) when reproject=True).  rows/out may be
        numpy arrays or CPU torch tensors (pinned for full copy speed)."""
        import torch
        if isinstance(rows, torch.Tensor):
            assert rows.device.type == "cpu" and rows.dtype == torch.float32 and rows.is_contiguous()
            rptr, S = ctypes.c_void_p(rows.data_ptr()), rows.shape[0]
        else:
            r = np.ascontiguousarray(rows, np.float32)
            rptr, S = r.ctypes.data_as(ctypes.c_void_p), r.shape[0]
        if out is None:
            out = np.empty((S, self.N0, self.N1), np.float32)
        mptr = ctypes.c_void_p(out.data_ptr()) if isinstance(out, torch.Tensor) else out.ctypes.data_as(ctypes.c_void_p)
        rp = np.empty((S, self.nx), np.float32) if reproject else None
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        st = ctypes.c_void_p(stream) if stream is not None else None
        _check(lib().icon_reconstruct_host(self._h, ctypes.byref(cfg), rptr, mptr,
                                           rp.ctypes.data_as(ctypes.c_void_p) if reproject else None, S, st))
        return (out, rp) if reproject else out

    def prepare_rhs_stack(self, stack, y0, S, skip_section=-1):
        """A^H W b of slices y0 .. y0+S-1 read from a device tilt stack
        (sections, ny, nx) float32 in file order; skip_section >= 0 leaves
        that section out (the stack then has one section more than the plan
        has tilts).  -> (S, N0, N1) complex64."""
        import torch
        stack = self._dev(stack, torch.float32)
        out = torch.empty((S, self.N0, self.N1), dtype=torch.complex64, device=self.device)
        _check(lib().icon_prepare_rhs_stack(self._h, _ptr(stack), stack.shape[1], int(y0), int(skip_section), _ptr(out),
                                            int(S), _stream()))
        return out

    def reconstruct_stack(self, stack, y0, S, iters=(0, 10, 0), data_type=1, threshold=0.03, skip_section=-1,
                          slices=True, reproject=False):
        """The solve of slices y0 .. y0+S-1 of a device tilt stack, on the
        device: slices (S, N1, N0) float32 in file layout (X fastest) and/or
        the reprojection (S, nx) at the plan's reprojection angle."""
        import torch
        stack = self._dev(stack, torch.float32)
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        m = torch.empty((S, self.N1, self.N0), dtype=torch.float32, device=self.device) if slices else None
        rp = torch.empty((S, self.nx), dtype=torch.float32, device=self.device) if reproject else None
        _check(lib().icon_reconstruct_stack(self._h, ctypes.byref(cfg), _ptr(stack), stack.shape[1], int(y0),
                                            int(skip_section), _ptr(m) if slices else None,
                                            _ptr(rp) if reproject else None, int(S), _stream()))
        return m, rp

    def reconstruct_stack_host(self, stack, y0, S, sink, iters=(0, 10, 0), data_type=1, threshold=0.03,
                               skip_section=-1, outputs=OUT_SLICES | OUT_REPROJECTION, ny=None):
        """icon_reconstruct_stack_host: `stack` is a device pointer (int) or a
        CUDA tensor (sections, ny, nx); sink(s0, count, slices, reproj) gets
        numpy views (count, N1, N0) / (count, nx) of the pinned buffers (valid
        only during the call; None when not requested) and returns 0 to go on."""
        import torch
        if isinstance(stack, torch.Tensor):
            stack = self._dev(stack, torch.float32)
            sptr, ny = _ptr(stack), stack.shape[1]
        else:
            sptr = ctypes.c_void_p(int(stack))
        N0, N1, nx = self.N0, self.N1, self.nx

        def _view(p, shape):
            if not p:
                return None
            n = int(np.prod(shape))
            return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_float)), shape=(n,)).reshape(shape)

        def _cb(_ctx, s0, count, hm, hr):
            try:
                return int(sink(s0, count, _view(hm, (count, N1, N0)), _view(hr, (count, nx))) or 0)
            except Exception:   # an exception cannot cross the C boundary
                return 1

        cb = BATCH_SINK(_cb)
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        _check(lib().icon_reconstruct_stack_host(self._h, ctypes.byref(cfg), sptr, int(ny), int(y0), int(skip_section),
                                                 int(S), int(outputs), cb, None, _stream()))

    TRACE_KINDS = ("xpass_fwd", "ypass_fwd", "interp_fin", "ypass_adj", "xpass_adj", "alpha", "update", "rows_fwd",
                   "layout", "row_adj", "ypass_toep", "ypass_toep_quad", "xtoep_fwd", "xtoep_mid")

    def trace(self, enable=True):
        _check(lib().icon_trace_enable(self._h, int(bool(enable))))

    def trace_read(self):
        """{kernel kind: (launches, total ms, algorithmic bytes)} since the last read."""
        n = len(self.TRACE_KINDS)
        cnt = (ctypes.c_int * n)()
        ms = (ctypes.c_double * n)()
        by = (ctypes.c_double * n)()
        _check(lib().icon_trace_read(self._h, ctypes.cast(cnt, ctypes.c_void_p), ctypes.cast(ms, ctypes.c_void_p),
                                     ctypes.cast(by, ctypes.c_void_p)))
        return {k: (int(cnt[i]), float(ms[i]), float(by[i])) for i, k in enumerate(self.TRACE_KINDS)}

    def device_error(self):
        """Reads and clears the plan's device error flag (0: none; 1: a
        bounded wait for the x-kernels' TMA loads ran out)."""
        v = ctypes.c_int(0)
        _check(lib().icon_plan_device_error(self._h, ctypes.byref(v)))
        return int(v.value)

    def launch_count(self):
        return int(lib().icon_launch_count(self._h))


class DeviceStack:
    """Rows y0 .. y0+S-1 of every section of a host tilt stack
    (sections, ny, nx) uploaded in one copy (icon_stack_upload) to device
    memory packed as (sections, S, nx); .ptr is the device address for the
    stack calls (with ny = S, y0 = 0)."""

    def __init__(self, h_stack, device=0, y0=0, S=None):
        st = np.ascontiguousarray(h_stack, np.float32)
        sec, ny, nx = st.shape
        S = ny - y0 if S is None else S
        p = ctypes.c_void_p()
        self._free = lib().icon_device_free
        _check(lib().icon_stack_upload(int(device), st.ctypes.data_as(ctypes.c_void_p), sec, ny, nx, int(y0), int(S),
                                       ctypes.byref(p), None))
        self.device, self.ptr, self.shape = int(device), p.value, (sec, S, nx)

    def close(self):
        if getattr(self, "ptr", None):
            self._free(self.device, ctypes.c_void_p(self.ptr))
            self.ptr = None

    __del__ = close


def host_alloc(nbytes):
    """Pinned host memory (icon_host_alloc) as a (pointer, free) pair."""
    p = ctypes.c_void_p()
    _check(lib().icon_host_alloc(int(nbytes), ctypes.byref(p)))
    return p.value, lambda: lib().icon_host_free(ctypes.c_void_p(p.value))


def weights(nx, tilts):
    """Density weights (ntilt, nx) of a tilt series given as in the .tlt
    file, as the plan weights its nodes (icon_weights; Weight, weight.cu:8-41)."""
    t = np.ascontiguousarray(np.asarray(tilts, np.float32))
    w = np.zeros((len(t), int(nx)), np.float32)
    _check(lib().icon_weights(int(nx), len(t), t.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p)))
    return w


class Series(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("thickness", ctypes.c_int), ("ntilt", ctypes.c_int),
                ("tilt_deg", ctypes.POINTER(ctypes.c_float)), ("slices", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("group", ctypes.c_int), ("chunk", ctypes.c_int), ("us_per_slice_iteration", ctypes.c_double),
                ("tuned", ctypes.c_int)]


class IconBatch:
    """Many tilt series of uneven shape reconstructed together
    (include/icon_batch.h): `series` is a list of (nx, thickness, tilts,
    slices).  tune: 0 = cache file or defaults, 1 = time shapes missing from
    the cache, 2 = also append them to the cache file."""

    def __init__(self, series, device=None, operator="toeplitz", tune_cache=None, tune=0):
        import torch
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device)
        self._tilts = [np.ascontiguousarray(np.asarray(t, np.float32)) for _, _, t, _ in series]
        arr = (Series * len(series))()
        for k, (nx, th, _, sl) in enumerate(series):
            t = self._tilts[k]
            arr[k] = Series(int(nx), int(th), len(t), t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(sl))
        self.shapes = [(int(nx), int(th) or int(nx), len(self._tilts[k]), int(sl))
                       for k, (nx, th, _, sl) in enumerate(series)]
        h = ctypes.c_void_p()
        self._destroy = lib().icon_batch_destroy
        _check(lib().icon_batch_create(arr, len(series), int(device), IconPlan.OPERATORS[operator],
                                       tune_cache.encode() if tune_cache else None, int(tune), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._destroy(h)
            self._h = None

    __del__ = close

    def tuning(self, k):
        t = Tuning()
        _check(lib().icon_batch_tuning(self._h, int(k), ctypes.byref(t)))
        return {"group": t.group, "chunk": t.chunk, "us_per_slice_iteration": t.us_per_slice_iteration,
                "tuned": t.tuned}

    def reconstruct(self, rows, iters=(0, 10, 0), data_type=1, threshold=0.03, out=None, concurrent=True):
        """rows: per series a host float32 array or tensor (slices, ntilt, nx),
        best pinned; returns per series (slices, N0, N1) float32 host tensors
        (pinned), or fills `out`."""
        import torch
        rows = [torch.as_tensor(np.ascontiguousarray(r, np.float32)) if not torch.is_tensor(r) else r.contiguous()
                for r in rows]
        if out is None:
            out = [torch.empty((sl, nx, th), dtype=torch.float32, pin_memory=True) for nx, th, _, sl in self.shapes]
        n = len(self.shapes)
        rp = (ctypes.c_void_p * n)(*[r.data_ptr() for r in rows])
        op = (ctypes.c_void_p * n)(*[o.data_ptr() for o in out])
        a, b, c = iters
        cfg = SolveCfg(int(a), int(b), int(c), int(data_type), float(threshold))
        _check(lib().icon_batch_reconstruct_host(self._h, ctypes.byref(cfg), rp, op, int(bool(concurrent))))
        return out
