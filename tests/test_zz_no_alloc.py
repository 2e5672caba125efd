"""GPU test of icon_rows_forward_noalloc, the entry point for callers that
cannot allocate device memory (a process whose pool allocator owns all device
memory, or a real-time loop that must not call cudaMalloc).  It must give the
same result as the plan-based icon_rows_forward, on consecutive calls that
share its static scratch array -- including a call right after one for a
different detector width, which leaves other tables behind in the array.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-5   # the tolerance of the other single-transform parity tests


def _noalloc():
    from feilab_b200 import icon
    L = icon.lib()
    f = L.icon_rows_forward_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return icon, f


def _call(f, rows, nx, nz):
    S = rows.shape[0]
    out = torch.full((S, nz * nx), float("nan"), dtype=torch.complex64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = f(ctypes.c_void_p(rows.data_ptr()), nx, nz, S, ctypes.c_void_p(out.data_ptr()), st)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_rows_match_plan_entry_point_on_consecutive_calls(golden):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    icon, f = _noalloc()
    for name in ("c", "a", "b"):
        z = golden[name]
        nx, nz, S = int(z["nx"]), len(z["tilts"]), int(z["S"])
        rows = torch.from_numpy(np.ascontiguousarray(z["rows"])).cuda()
        plan = icon.IconPlan(nx, int(z["thickness"]), z["tilts"], capacity=S)
        ref = plan.rows_forward(rows).cpu().numpy()
        first = _call(f, rows, nx, nz)
        second = _call(f, rows, nx, nz)
        for out in (first, second):
            assert np.isfinite(out.view(np.float32)).all()
            for s in range(S):
                assert rel_l2(out[s], ref[s]) < TOL_STAGE, (name, s)
                assert rel_l2(out[s], z["ref_b"][s]) < TOL_STAGE, (name, s)
        plan.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    icon, f = _noalloc()
    rows = torch.zeros((1, 2, 16), dtype=torch.float32, device="cuda")
    out = torch.zeros((1, 32), dtype=torch.complex64, device="cuda")
    rc = f(ctypes.c_void_p(rows.data_ptr()), 8192, 2, 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"nx must be" in icon.lib().icon_last_error()
