"""CPU checks of the native boundary: the library builds for sm_100a, loads
without a GPU, and exports every function include/*.h declares."""
import ctypes
import os
import re

from conftest import ROOT


def _declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\*?\s*(icon_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared_functions()
    for n in ("icon_plan_create", "icon_nufft_forward", "icon_nufft_adjoint", "icon_solve", "icon_last_error"):
        assert n in names


def test_library_loads_and_exports_every_declared_symbol():
    from feilab_b200 import build
    lib_path = build.build_lib()
    L = ctypes.CDLL(lib_path)
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    L.icon_last_error.restype = ctypes.c_char_p
    assert L.icon_last_error() == b""


def test_plan_create_without_gpu_fails_cleanly():
    # With no device the call must return an error status, not abort.
    import torch
    if torch.cuda.is_available():
        return
    from feilab_b200 import icon
    import numpy as np
    try:
        icon.IconPlan(16, 16, np.array([-10, 0, 10], np.float32), capacity=1, device=0)
    except icon.IconError as e:
        assert "status" in str(e)
    else:
        raise AssertionError("plan creation without a GPU should fail")


def test_shipped_warm_start_weights_match_the_network():
    # The trained warm-start network shipped with the library has exactly the
    # parameter count of the network the library builds.
    from feilab_b200 import warmstart
    params, gain, meta = warmstart.load_weights()
    assert params.size == warmstart.param_count()
    assert gain > 0 and meta["nx"] == 1024 and meta["thickness"] == 300


def test_raw_weights_file_layout(tmp_path):
    # The weights file icon-gpu --warm-start reads (icon_ws_load): magic,
    # uint64 parameter count, float32 gain, then the FP32 parameters, for
    # both shipped networks (1024x300 and the 512x256 one of the
    # learned-start workload).
    import struct
    import numpy as np
    from feilab_b200 import warmstart
    for nx, th in ((1024, 300), (512, 256)):
        params, gain, meta = warmstart.load_weights(nx=nx, thickness=th)
        assert params.size == warmstart.param_count() and (meta["nx"], meta["thickness"]) == (nx, th)
        f = tmp_path / f"w{nx}.bin"
        warmstart.save_raw(str(f), params, gain)
        raw = f.read_bytes()
        assert raw[:8] == b"ICONWSB1"
        n, g = struct.unpack("<Qf", raw[8:20])
        assert n == params.size and abs(g - gain) <= 1e-6 * abs(gain)
        assert np.array_equal(np.frombuffer(raw[20:], "<f4"), params)
