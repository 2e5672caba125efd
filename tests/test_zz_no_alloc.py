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


@pytest.mark.parametrize("nx,nz,S", [
    (8, 5, 1),       # n = 16, the smallest FFT; one slice per group, a one-thread block
    (8, 5, 3),
    (1024, 9, 9),    # groups of 8 slices, 128 KiB of dynamic shared memory
    (4096, 3, 1),    # n = 8192: one slice per group, 512 threads, 64 KiB
    (4096, 3, 3),    # n = 8192: two slices per group, 1024 threads, 128 KiB
])
def test_noalloc_rows_match_plan_entry_point_at_extreme_sizes(nx, nz, S):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    icon, f = _noalloc()
    rng = np.random.default_rng(nx * 131 + S)
    tilts = np.linspace(-50.0, 50.0, nz).astype(np.float32)
    rows = torch.from_numpy(rng.standard_normal((S, nz, nx)).astype(np.float32)).cuda()
    plan = icon.IconPlan(nx, 8, tilts, capacity=S)
    ref = plan.rows_forward(rows).cpu().numpy()
    plan.close()
    for _ in range(2):
        out = _call(f, rows, nx, nz)
        assert np.isfinite(out.view(np.float32)).all()
        for s in range(S):
            assert rel_l2(out[s], ref[s]) < TOL_STAGE, (nx, S, s)


def test_noalloc_second_call_allocates_no_device_memory():
    """After the first call on a device has loaded the library's device code
    (which holds the scratch array), further calls leave the device's free
    memory unchanged: they allocate nothing."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    icon, f = _noalloc()
    nx, nz, S = 512, 7, 4
    rows = torch.from_numpy(np.random.default_rng(5).standard_normal((S, nz, nx)).astype(np.float32)).cuda()
    out = torch.empty((S, nz * nx), dtype=torch.complex64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (ctypes.c_void_p(rows.data_ptr()), nx, nz, S, ctypes.c_void_p(out.data_ptr()), st)
    assert f(*args) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert f(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    icon, f = _noalloc()
    rows = torch.zeros((1, 2, 16), dtype=torch.float32, device="cuda")
    out = torch.zeros((1, 32), dtype=torch.complex64, device="cuda")
    rc = f(ctypes.c_void_p(rows.data_ptr()), 8192, 2, 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"nx must be" in icon.lib().icon_last_error()
