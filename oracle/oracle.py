"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module as the checker.  The product path
(feilab_b200) never imports it.

The oracle restates the ICON-GPU v1.2.9 hot path on the CPU (see
oracle/icon_oracle_core.c for the reference file:line of every routine).
Image arrays are (N0, N1) with the thickness index Y fastest, exactly the
reference's device layout; node arrays are (M,) complex with node j = tilt*nx + k.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


def _declare(L):
    fp = ctypes.POINTER(ctypes.c_float)
    for sfx in ("_f64", "_f32"):
        getattr(L, "ora_plan_create" + sfx).argtypes = [_I, _I, _I, fp, ctypes.POINTER(_P)]
        getattr(L, "ora_plan_create_line" + sfx).argtypes = [_I, _I, _F, ctypes.POINTER(_P)]
        getattr(L, "ora_plan_create_w" + sfx).argtypes = [_I, _I, _I, fp, _I, ctypes.POINTER(_P)]
        getattr(L, "ora_plan_create_line_w" + sfx).argtypes = [_I, _I, _F, _I, ctypes.POINTER(_P)]
        getattr(L, "ora_plan_destroy" + sfx).argtypes = [_P]
        getattr(L, "ora_plan_dims" + sfx).argtypes = [_P, ctypes.POINTER(_I)]
        getattr(L, "ora_plan_geometry" + sfx).argtypes = [_P, _P, _P, _P]
        getattr(L, "ora_plan_windows" + sfx).argtypes = [_P] * 7
        getattr(L, "ora_nufft_forward" + sfx).argtypes = [_P, _P, _I, _P]
        getattr(L, "ora_nufft_adjoint" + sfx).argtypes = [_P, _P, _P]
        getattr(L, "ora_rows_forward" + sfx).argtypes = [_P, _P, _P]
        getattr(L, "ora_row_adjoint" + sfx).argtypes = [_P, _P, _P]
        getattr(L, "ora_rhs" + sfx).argtypes = [_P, _P, _P]
        getattr(L, "ora_solve" + sfx).argtypes = [_P, _P, _I, _I, _I, _I, _F, _P, _P, _P]
        getattr(L, "ora_reproject" + sfx).argtypes = [_P, _P, _P, _P]
        getattr(L, "ora_reconstruct" + sfx).argtypes = [_P, _P, _I, _I, _I, _I, _I, _F, _P, _I]
        getattr(L, "ora_reconstruct" + sfx).restype = _I
        getattr(L, "ora_rhs_batch" + sfx).argtypes = [_P, _P, _I, _P, _I]
        getattr(L, "ora_rhs_batch" + sfx).restype = _I
        getattr(L, "ora_solve_batch" + sfx).argtypes = [_P, _P, _I, _I, _I, _I, _I, _F, _P, _I]
        getattr(L, "ora_solve_batch" + sfx).restype = _I
        getattr(L, "ora_ndft_forward" + sfx).argtypes = [_P, _P, _I, _P]
        getattr(L, "ora_ndft_adjoint" + sfx).argtypes = [_P, _P, _P]
    L.ora_grid_params.argtypes = [_I, fp, ctypes.POINTER(_I), fp, fp]


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def grid_params(N: int):
    """(theta, n, b, bf) of one dimension, MainCode.cu:66-71 and NU:471-476."""
    th, b, bf = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    n = ctypes.c_int()
    lib().ora_grid_params(N, ctypes.byref(th), ctypes.byref(n), ctypes.byref(b), ctypes.byref(bf))
    return th.value, n.value, b.value, bf.value


class OraclePlan:
    """One tilt series (nx, thickness, tilt angles as read from the .tlt file).

    precision: "f64" (the FP64 oracle) or "f32" (float rounding as the
    reference, radix-2 FFT in place of cuFFT).  window: "gauss6" (the
    reference's Gaussian window) or "kb4" (Kaiser-Bessel, half-width 4).
    """

    WINDOWS = {"gauss6": 0, "kb4": 1}

    def __init__(self, nx: int, thickness: int, tilts, precision: str = "f64", line_angle=None, window="gauss6"):
        self.sfx = "_" + precision
        self.real = np.float64 if precision == "f64" else np.float32
        self.cplx = np.complex128 if precision == "f64" else np.complex64
        h = ctypes.c_void_p()
        L = lib()
        wk = self.WINDOWS[window]
        self.window = window
        if line_angle is not None:
            rc = getattr(L, "ora_plan_create_line_w" + self.sfx)(nx, thickness, ctypes.c_float(line_angle), wk,
                                                                 ctypes.byref(h))
        else:
            t = np.ascontiguousarray(np.asarray(tilts, dtype=np.float32))
            rc = getattr(L, "ora_plan_create_w" + self.sfx)(nx, thickness, len(t),
                                                            t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), wk,
                                                            ctypes.byref(h))
        if rc != 0:
            raise ValueError(f"oracle plan rejected (nx={nx}, thickness={thickness})")
        self._h = h
        d = (ctypes.c_int * 6)()
        getattr(L, "ora_plan_dims" + self.sfx)(h, d)
        self.N0, self.N1, self.n0, self.n1, self.M, self.nz = list(d)
        self.nx = nx

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            getattr(lib(), "ora_plan_destroy" + self.sfx)(h)
            self._h = None

    def _fn(self, name):
        return getattr(lib(), name + self.sfx)

    def geometry(self):
        xy = np.zeros((self.M, 2), np.float32)
        w = np.zeros(self.M, np.float32)
        prm = np.zeros(6, np.float32)
        self._fn("ora_plan_geometry")(self._h, _ptr(xy), _ptr(w), _ptr(prm))
        return xy, w, prm

    def windows(self):
        T = 14
        phix = np.zeros((self.M, T), self.real)
        phiy = np.zeros((self.M, T), self.real)
        ix = np.zeros((self.M, T), np.int32)
        iy = np.zeros((self.M, T), np.int32)
        cx = np.zeros(self.N0, self.real)
        cy = np.zeros(self.N1, self.real)
        self._fn("ora_plan_windows")(self._h, _ptr(phix), _ptr(ix), _ptr(phiy), _ptr(iy), _ptr(cx), _ptr(cy))
        return phix, ix, phiy, iy, cx, cy

    def forward(self, img: np.ndarray) -> np.ndarray:
        """A img: (N0, N1) real or complex image -> (M,) complex."""
        is_real = not np.iscomplexobj(img)
        x = np.ascontiguousarray(img, dtype=self.real if is_real else self.cplx)
        f = np.zeros(self.M, self.cplx)
        self._fn("ora_nufft_forward")(self._h, _ptr(x), int(is_real), _ptr(f))
        return f

    def adjoint(self, f: np.ndarray) -> np.ndarray:
        """A^H f: (M,) complex -> (N0, N1) complex."""
        x = np.ascontiguousarray(f, dtype=self.cplx)
        out = np.zeros((self.N0, self.N1), self.cplx)
        self._fn("ora_nufft_adjoint")(self._h, _ptr(x), _ptr(out))
        return out

    def rows_forward(self, rows: np.ndarray) -> np.ndarray:
        """(nz, nx) projection rows -> b (M,) complex."""
        r = np.ascontiguousarray(rows, dtype=np.float32)
        b = np.zeros(self.M, self.cplx)
        self._fn("ora_rows_forward")(self._h, _ptr(r), _ptr(b))
        return b

    def row_adjoint(self, f: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(f, dtype=self.cplx)
        out = np.zeros(self.nx, self.cplx)
        self._fn("ora_row_adjoint")(self._h, _ptr(x), _ptr(out))
        return out

    def rhs(self, rows: np.ndarray) -> np.ndarray:
        """A^H W b for one slice's projection rows -> (N0, N1) complex."""
        r = np.ascontiguousarray(rows, dtype=np.float32)
        out = np.zeros((self.N0, self.N1), self.cplx)
        self._fn("ora_rhs")(self._h, _ptr(r), _ptr(out))
        return out

    def solve(self, Ahwb, iters=(0, 10, 0), data_type=1, threshold=0.03, m0=None, history=False):
        a, b, c = iters
        A = np.ascontiguousarray(Ahwb, dtype=self.cplx)
        m = np.zeros((self.N0, self.N1), self.real) if m0 is None else np.array(m0, dtype=self.real, order="C")
        n = a + b + c
        al = np.zeros(max(n, 1), np.float64)
        rt = np.zeros(max(n, 1), np.float64)
        self._fn("ora_solve")(self._h, _ptr(A), a, b, c, data_type, ctypes.c_float(threshold), _ptr(m), _ptr(al), _ptr(rt))
        if history:
            return m, al[:n], rt[:n]
        return m

    def reproject(self, line_plan: "OraclePlan", m: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(m, dtype=self.real)
        out = np.zeros(self.nx, self.real)
        self._fn("ora_reproject")(line_plan._h, self._h, _ptr(x), _ptr(out))
        return out

    def reconstruct(self, rows: np.ndarray, iters=(0, 10, 0), data_type=1, threshold=0.03, nthreads=0):
        """rows: (S, nz, nx) -> m (S, N0, N1); OpenMP over slices."""
        r = np.ascontiguousarray(rows, dtype=np.float32)
        S = r.shape[0]
        m = np.zeros((S, self.N0, self.N1), self.real)
        a, b, c = iters
        used = self._fn("ora_reconstruct")(self._h, _ptr(r), S, a, b, c, data_type, ctypes.c_float(threshold), _ptr(m), nthreads)
        self.threads_used = used
        return m

    def rhs_batch(self, rows: np.ndarray, nthreads=0) -> np.ndarray:
        """rows (S, nz, nx) -> A^H W b (S, N0, N1); OpenMP over slices."""
        r = np.ascontiguousarray(rows, dtype=np.float32)
        out = np.zeros((r.shape[0], self.N0, self.N1), self.cplx)
        self.threads_used = self._fn("ora_rhs_batch")(self._h, _ptr(r), r.shape[0], _ptr(out), nthreads)
        return out

    def solve_batch(self, Ahwb, m, iters, data_type, threshold, nthreads=0):
        """ICON iterations (a, b, c) on every slice, in place: m (S, N0, N1)
        holds the start values and receives the results; OpenMP over slices."""
        A = np.ascontiguousarray(Ahwb, dtype=self.cplx)
        assert m.dtype == self.real and m.flags["C_CONTIGUOUS"] and m.shape == A.shape
        a, b, c = iters
        self.threads_used = self._fn("ora_solve_batch")(self._h, _ptr(A), A.shape[0], a, b, c, data_type,
                                                        ctypes.c_float(threshold), _ptr(m), nthreads)
        return m

    def ndft_forward(self, img: np.ndarray) -> np.ndarray:
        is_real = not np.iscomplexobj(img)
        x = np.ascontiguousarray(img, dtype=np.float64 if is_real else np.complex128)
        f = np.zeros(self.M, np.complex128)
        self._fn("ora_ndft_forward")(self._h, _ptr(x), int(is_real), _ptr(f))
        return f

    def ndft_adjoint(self, f: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(f, dtype=np.complex128)
        out = np.zeros((self.N0, self.N1), np.complex128)
        self._fn("ora_ndft_adjoint")(self._h, _ptr(x), _ptr(out))
        return out
