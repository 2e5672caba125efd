"""GPU versions of the reference's companion tools against the reference
tools' own outputs (fixtures in tests/golden written by the reference
binaries built from their sources).

Pre-processing: mode subtraction uses the reference's arithmetic step by step
(double min / max / bin / mode, float result), so it is compared bit for
bit; the variance normalisation sums in double in another order, so within
2e-6 of the largest value.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu
TOL_NORM = 2e-6


@pytest.mark.parametrize("name", ["p1", "p2"])
def test_preprocess_matches_reference_tool(name):
    from feilab_b200 import tools
    z = load_golden("preprocess")
    st = torch.from_numpy(z[name + "_stack"]).cuda()
    got = tools.preprocess(st).cpu().numpy()
    np.testing.assert_array_equal(got, z[name + "_mode_only"])
    got = tools.preprocess(st, z[name + "_tilts"], int(z[name + "_thickness"])).cpu().numpy()
    ref = z[name + "_normalized"]
    assert np.max(np.abs(got - ref)) <= TOL_NORM * np.max(np.abs(ref))


def test_preprocess_in_place():
    from feilab_b200 import tools
    z = load_golden("preprocess")
    st = torch.from_numpy(z["p2_stack"]).cuda()
    tools.preprocess(st, z["p2_tilts"], int(z["p2_thickness"]), out=st)
    ref = z["p2_normalized"]
    assert np.max(np.abs(st.cpu().numpy() - ref)) <= TOL_NORM * np.max(np.abs(ref))


def test_preprocess_tool_matches_reference_tool(tmp_path):
    from feilab_b200 import mrc
    z = load_golden("preprocess")
    fin, tlt, fout = tmp_path / "in.mrc", tmp_path / "t.tlt", tmp_path / "out.mrc"
    mrc.write(str(fin), z["p1_stack"])
    mrc.write_tlt(str(tlt), z["p1_tilts"])
    exe = os.path.join(ROOT, "feilab_b200", "icon-preprocess")
    p = subprocess.run([exe, "-i", str(fin), "-t", str(tlt), "-th", str(int(z["p1_thickness"])), "-o", str(fout)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    h, d = mrc.read(str(fout))
    ref = z["p1_normalized"]
    assert d.shape == ref.shape
    assert np.max(np.abs(d - ref)) <= TOL_NORM * np.max(np.abs(ref))
    href = np.frombuffer(z["p1_header"].tobytes(), mrc.HEADER_DTYPE)[0]
    for f in ("nx", "ny", "nz", "mode"):
        assert int(h[f]) == int(href[f])
    for f in ("amin", "amax", "amean"):
        assert abs(float(h[f]) - float(href[f])) <= 1e-4 * max(1.0, abs(float(href[f])))


def test_preprocess_rejects_bad_input():
    from feilab_b200 import tools
    from feilab_b200.icon import IconError
    with pytest.raises(IconError):
        tools.preprocess(torch.zeros((2, 3, 4), device="cuda", dtype=torch.float64))


# ---------------------------------------------------------------- ICONMask3
MASK_CASES = {
    # name: (thickness, zshift, radius or None (from the FRC files), gauss width or None, masked)
    "frc": (64, 0, None, None, True),
    "radius": (64, 0, 12, 6, True),
    "crop": (40, 5, 15, None, True),
    "nomask": (48, 0, None, None, False),
}
TOL_MASK = 1e-5        # relative L2: our float FFT against cuFFT's


@pytest.mark.parametrize("name", ["frc", "radius", "crop"])
def test_mask_matches_reference_tool(name):
    from feilab_b200 import tools
    z = load_golden("mask")
    th, zs, radius, gw, _ = MASK_CASES[name]
    mids = torch.from_numpy(z["mids"]).cuda()
    n = mids.shape[-1]
    r05, r03, ex = tools.mask_radius(n, z["tilts"], radius, z["crossV_frc"][:, 1], z["fullRec_frc"][:, 1])
    m = tools.Mask(n, z["tilts"], r05, r03, ex, gw, capacity=8)
    got = m.apply(mids, n // 2 - th // 2 + zs, th).cpu().numpy()
    ref = z["vol_" + name]
    assert got.shape == ref.shape
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL_MASK


@pytest.mark.parametrize("name", list(MASK_CASES))
def test_mask_tool_matches_reference_tool(name, tmp_path):
    from feilab_b200 import mrc
    z = load_golden("mask")
    th, zs, radius, gw, masked = MASK_CASES[name]
    rec = tmp_path / "reconstruction"
    rec.mkdir()
    hdr = z["mid_header"].tobytes()
    for s, sl in enumerate(z["mids"]):
        (rec / f"mid{s:05d}.mrc").write_bytes(hdr + np.ascontiguousarray(sl, np.float32).tobytes())
    tlt, vol = tmp_path / "t.tlt", tmp_path / "vol.mrc"
    mrc.write_tlt(str(tlt), z["tilts"])
    np.savetxt(tmp_path / "crossV.frc", z["crossV_frc"], fmt="%f")
    np.savetxt(tmp_path / "fullRec.frc", z["fullRec_frc"], fmt="%f")
    args = ["-i", str(rec), "-s", f"0,{len(z['mids']) - 1}", "-t", str(tlt), "-o", str(vol), "-th", str(th)]
    if zs:
        args += ["-z", str(zs)]
    if not masked:
        args += ["-nm", "1"]
    elif radius is None:
        args += ["-cf", str(tmp_path / "crossV.frc"), "-ff", str(tmp_path / "fullRec.frc")]
    else:
        args += ["-r", str(radius)]
    if gw:
        args += ["-gw", str(gw)]
    exe = os.path.join(ROOT, "feilab_b200", "icon-mask")
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=120)
    assert p.returncode == (0 if masked else 1), p.stdout + p.stderr
    h, d = mrc.read(str(vol))
    ref = z["vol_" + name]
    assert d.shape == ref.shape
    if masked:
        assert np.linalg.norm(d - ref) / np.linalg.norm(ref) < TOL_MASK
    else:
        np.testing.assert_array_equal(d, ref)
    href = np.frombuffer(z["hdr_" + name].tobytes(), mrc.HEADER_DTYPE)[0]
    for f in ("nx", "ny", "nz", "mode"):
        assert int(h[f]) == int(href[f])
    for f in ("amin", "amax"):
        assert abs(float(h[f]) - float(href[f])) <= 1e-4 * max(1.0, abs(float(href[f])))
