"""The icon-gpu command-line tool against the reference ICON-GPU run.

The golden "cli" case holds what the reference tool wrote for a 64-pixel,
25-tilt stack (slices 0..3, thickness 40, -iter 1,5,1): the slice files
reconstruction/midNNNNN.mrc (ICONGPU.cu:330-366, saveMRC_real.cu:33-56) and the
crossValidation outputs (GroundTruth / reprojection MRCs and the smoothed FRC
curves, ICONGPU.cu:468-592).  The same stack and tilt file are written here,
the tool is run on them and every file is compared: headers field by field,
data within the solve tolerance, FRC curves within an absolute tolerance.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "feilab_b200", "icon-gpu")
TOL_SOLVE = 1e-4      # relative L2, as the solve parity tests
TOL_FRC = 2e-3        # absolute, per FRC ring
STAT_FIELDS = ("amin", "amax", "amean", "rms")


def _run(args, cwd):
    return subprocess.run([TOOL] + args, cwd=cwd, capture_output=True, text=True, timeout=300)


def _mrc_from_bytes(raw, tmp_path, name):
    from feilab_b200 import mrc
    p = tmp_path / name
    p.write_bytes(raw)
    return mrc.read(str(p))


def _compare_headers(h, hr):
    for f in h.dtype.names:
        if f in STAT_FIELDS:
            np.testing.assert_allclose(float(h[f]), float(hr[f]), rtol=1e-3, atol=1e-5, err_msg=f)
        else:
            assert np.array_equal(h[f], hr[f]), f


def test_cli_usage_errors(tmp_path):
    p = _run(["-i", "missing.mrc"], str(tmp_path))
    assert p.returncode != 0
    assert "parameter error!" in p.stdout


@pytest.mark.gpu
def test_cli_matches_reference_tool(golden, tmp_path):
    from feilab_b200 import mrc
    z = golden["cli"]
    nx, th, S = int(z["nx"]), int(z["thickness"]), int(z["S"])
    stack, tlt, out = tmp_path / "stack.mrc", tmp_path / "cli.tlt", tmp_path / "res"
    mrc.write_tilt_series(str(stack), z["rows"])
    mrc.write_tlt(str(tlt), z["tilts"])
    out.mkdir()
    a, b, c = (int(v) for v in z["sched"])
    p = _run(["-i", str(stack), "-t", str(tlt), "-o", str(out), "-s", f"0,{S - 1}", "-iter", f"{a},{b},{c}",
              "-d", str(int(z["data_type"])), "-thr", str(float(z["threshold"])), "-g", "0", "-thi", str(th)],
             str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    assert "ICON-GPU finish!" in p.stdout
    for s in range(S):
        assert f"slice {s} finished" in p.stdout
        h, d = mrc.read(str(out / "reconstruction" / f"mid{s:05d}.mrc"))
        hr, dr = _mrc_from_bytes(z[f"cli_mid{s:05d}"].tobytes(), tmp_path, f"ref{s}.mrc")
        _compare_headers(h, hr)
        assert d.shape == dr.shape == (1, th, nx)
        assert rel_l2(d[0], dr[0]) < TOL_SOLVE, s
    for fn in ("GroundTruth.mrc", "fullRec_reProjection.mrc", "crossV_reprojection.mrc"):
        h, d = mrc.read(str(out / "crossValidation" / fn))
        hr, dr = _mrc_from_bytes(z["cli_" + fn.replace(".", "_")].tobytes(), tmp_path, "ref_" + fn)
        _compare_headers(h, hr)
        assert d.shape == dr.shape
        if fn == "GroundTruth.mrc":
            np.testing.assert_array_equal(d, dr)
        else:
            assert rel_l2(d, dr) < TOL_SOLVE, fn
    for fn in ("fullRec.frc", "crossV.frc"):
        got = np.loadtxt(str(out / "crossValidation" / fn))
        ref = np.loadtxt(z["cli_" + fn.replace(".", "_")].tobytes().decode().splitlines())
        assert got.shape == ref.shape == (nx // 2, 2)
        np.testing.assert_array_equal(got[:, 0], ref[:, 0])
        np.testing.assert_allclose(got[:, 1], ref[:, 1], atol=TOL_FRC, err_msg=fn)


@pytest.mark.gpu
def test_cli_volume_output(golden, tmp_path):
    # --volume writes the slices as one MRC (sections = slices, X fastest), the
    # same values as the per-slice files.
    from feilab_b200 import mrc
    z = golden["cli"]
    nx, th, S = int(z["nx"]), int(z["thickness"]), int(z["S"])
    stack, tlt, out = tmp_path / "stack.mrc", tmp_path / "cli.tlt", tmp_path / "res"
    mrc.write_tilt_series(str(stack), z["rows"])
    mrc.write_tlt(str(tlt), z["tilts"])
    out.mkdir()
    vol = tmp_path / "vol.mrc"
    p = _run(["-i", str(stack), "-t", str(tlt), "-o", str(out), "-s", f"0,{S - 1}", "-iter", "1,5,1", "-d", "2",
              "-thr", "0", "-g", "0", "-thi", str(th), "-skipCV", "1", "--volume", str(vol)], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    h, v = mrc.read(str(vol))
    assert v.shape == (S, th, nx)
    for s in range(S):
        _, d = mrc.read(str(out / "reconstruction" / f"mid{s:05d}.mrc"))
        np.testing.assert_array_equal(v[s], d[0])


@pytest.mark.gpu
def test_cli_leave_one_out(golden, tmp_path):
    # --loo writes one FRC curve per omitted tilt; the curve of the tilt the
    # reference cross-validates equals the tool's own crossV.frc (the same
    # left-out solve, run in the batched schedule).
    from feilab_b200 import mrc
    from conftest import min_abs_tilt_index
    z = golden["cli"]
    nx, th, S = int(z["nx"]), int(z["thickness"]), int(z["S"])
    nz = len(z["tilts"])
    stack, tlt, out = tmp_path / "stack.mrc", tmp_path / "cli.tlt", tmp_path / "res"
    mrc.write_tilt_series(str(stack), z["rows"])
    mrc.write_tlt(str(tlt), z["tilts"])
    out.mkdir()
    a, b, c = (int(v) for v in z["sched"])
    p = _run(["-i", str(stack), "-t", str(tlt), "-o", str(out), "-s", f"0,{S - 1}", "-iter", f"{a},{b},{c}",
              "-d", str(int(z["data_type"])), "-thr", str(float(z["threshold"])), "-g", "0", "-thi", str(th),
              "--loo", "--batch", "8"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    cv = out / "crossValidation"
    files = sorted((cv / "loo").glob("tilt*.frc"))
    assert len(files) == nz
    omit = min_abs_tilt_index(z["tilts"])
    got = np.loadtxt(str(cv / "loo" / f"tilt{omit:03d}.frc"))
    ref = np.loadtxt(str(cv / "crossV.frc"))
    np.testing.assert_array_equal(got[:, 0], ref[:, 0])
    np.testing.assert_allclose(got[:, 1], ref[:, 1], atol=1e-4)
    summary = np.loadtxt(str(cv / "loo_summary.txt"))
    assert summary.shape == (nz, 4)
    np.testing.assert_allclose(summary[:, 1], z["tilts"], atol=1e-5)
    assert np.all(summary[:, 3] == a + b + c)


def _cli_case(golden, tmp_path, name="res", sched=None):
    from feilab_b200 import mrc
    z = golden["cli"]
    stack, tlt, out = tmp_path / "stack.mrc", tmp_path / "cli.tlt", tmp_path / name
    if not stack.exists():
        mrc.write_tilt_series(str(stack), z["rows"])
        mrc.write_tlt(str(tlt), z["tilts"])
    out.mkdir()
    a, b, c = sched or (int(v) for v in z["sched"])
    base = ["-i", str(stack), "-t", str(tlt), "-o", str(out), "-s", f"0,{int(z['S']) - 1}", "-iter", f"{a},{b},{c}",
            "-d", str(int(z["data_type"])), "-thr", str(float(z["threshold"])), "-g", "0", "-thi",
            str(int(z["thickness"]))]
    return z, out, base


@pytest.mark.gpu
def test_cli_resume_keeps_finished_slices(golden, tmp_path):
    # A run whose slice files are partly there (an interrupted run) resumed
    # with --resume: the missing slices are reconstructed, the others read
    # back; every output file equals an uninterrupted run's byte for byte
    # (the reprojections of the read-back slices are recomputed from them).
    z, out, base = _cli_case(golden, tmp_path)
    S = int(z["S"])
    p = _run(base, str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    first = {f: (out / f).read_bytes() for f in
             [f"reconstruction/mid{s:05d}.mrc" for s in range(S)] +
             [f"crossValidation/{n}" for n in ("fullRec_reProjection.mrc", "crossV_reprojection.mrc", "fullRec.frc",
                                               "crossV.frc")]}
    (out / "reconstruction" / "mid00001.mrc").unlink()
    (out / "reconstruction" / f"mid{S - 1:05d}.mrc").write_bytes(b"truncated")
    for n in ("fullRec_reProjection.mrc", "crossV_reprojection.mrc", "fullRec.frc", "crossV.frc"):
        (out / "crossValidation" / n).unlink()
    p = _run(base + ["--resume"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"resume: {S - 2} of {S} slices" in p.stdout
    assert "slice 1 finished" in p.stdout and "slice 0 finished" not in p.stdout
    for f, data in first.items():
        assert (out / f).read_bytes() == data, f


@pytest.mark.gpu
def test_cli_toeplitz_operator_and_tolerance(golden, tmp_path):
    # --operator toeplitz reconstructs within the parity bar of the default
    # (NUFFT) run; --tol with a loose tolerance stops the ICON phase early
    # (slices differ, but stay close).
    from feilab_b200 import mrc
    sched = (1, 40, 1)
    z, out, base = _cli_case(golden, tmp_path, "nufft", sched)
    S, th, nx = int(z["S"]), int(z["thickness"]), int(z["nx"])
    assert _run(base + ["-skipCV", "1"], str(tmp_path)).returncode == 0
    zt, out_t, base_t = _cli_case(golden, tmp_path, "toep", sched)
    p = _run(base_t + ["-skipCV", "1", "--operator", "toeplitz"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    _, out_l, base_l = _cli_case(golden, tmp_path, "tol", sched)
    p = _run(base_l + ["-skipCV", "1", "--tol", "0.5"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    for s in range(S):
        _, d = mrc.read(str(out / "reconstruction" / f"mid{s:05d}.mrc"))
        _, dt = mrc.read(str(out_t / "reconstruction" / f"mid{s:05d}.mrc"))
        _, dl = mrc.read(str(out_l / "reconstruction" / f"mid{s:05d}.mrc"))
        assert d.shape == dt.shape == dl.shape == (1, th, nx)
        assert rel_l2(dt[0], d[0]) < TOL_SOLVE, s
        assert 0 < rel_l2(dl[0], d[0]) < 0.5, s
    p = _run(base + ["-skipCV", "1", "--operator", "other"], str(tmp_path))
    assert p.returncode != 0 and "parameter error!" in p.stdout


@pytest.mark.gpu
def test_cli_kaiser_bessel_window(golden, tmp_path):
    # --window kb4 reconstructs within the parity bar of the default
    # (Gaussian) run, cross-validation files included; an unknown window is
    # a parameter error.
    from feilab_b200 import mrc
    sched = (1, 40, 1)
    z, out, base = _cli_case(golden, tmp_path, "gauss", sched)
    S = int(z["S"])
    assert _run(base, str(tmp_path)).returncode == 0
    _, out_k, base_k = _cli_case(golden, tmp_path, "kb", sched)
    p = _run(base_k + ["--window", "kb4"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    for s in range(S):
        _, d = mrc.read(str(out / "reconstruction" / f"mid{s:05d}.mrc"))
        _, dk = mrc.read(str(out_k / "reconstruction" / f"mid{s:05d}.mrc"))
        assert d.shape == dk.shape
        assert rel_l2(dk[0], d[0]) < TOL_SOLVE, s
    for n in ("fullRec_reProjection.mrc", "crossV_reprojection.mrc"):
        _, r = mrc.read(str(out / "crossValidation" / n))
        _, rk = mrc.read(str(out_k / "crossValidation" / n))
        assert rel_l2(rk, r) < TOL_SOLVE, n
    p = _run(base + ["-skipCV", "1", "--window", "kb6"], str(tmp_path))
    assert p.returncode != 0 and "parameter error!" in p.stdout


@pytest.mark.gpu
def test_cli_warm_start(golden, tmp_path):
    # --warm-start FILE: the shipped network's weights exported to the raw
    # file format; every slice is either accepted from its warm start or
    # solved again from zero, the counts are printed, and the slices stay
    # finite and near the cold run's.  A file that is not a weights file is
    # refused.
    from feilab_b200 import mrc, warmstart
    params, gain, _ = warmstart.load_weights()
    wfile = tmp_path / "net.bin"
    warmstart.save_raw(str(wfile), params, gain)
    sched = (2, 40, 2)
    z, out, base = _cli_case(golden, tmp_path, "cold", sched)
    S = int(z["S"])
    assert _run(base + ["-skipCV", "1"], str(tmp_path)).returncode == 0
    _, out_w, base_w = _cli_case(golden, tmp_path, "warm", sched)
    p = _run(base_w + ["-skipCV", "1", "--warm-start", str(wfile), "--tol", "0.05"], str(tmp_path))
    assert p.returncode == 0, p.stdout + p.stderr
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("warm start:")]
    assert line and f"of {S} slices accepted" in line[0], p.stdout
    for s in range(S):
        _, d = mrc.read(str(out / "reconstruction" / f"mid{s:05d}.mrc"))
        _, dw = mrc.read(str(out_w / "reconstruction" / f"mid{s:05d}.mrc"))
        assert np.all(np.isfinite(dw))
        assert rel_l2(dw[0], d[0]) < 0.5, s
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not weights")
    _, out_b, base_b = _cli_case(golden, tmp_path, "bad", sched)
    p = _run(base_b + ["-skipCV", "1", "--warm-start", str(bad)], str(tmp_path))
    assert p.returncode != 0 and "warm start" in p.stdout
