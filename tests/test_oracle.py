"""CPU tests of the oracle: pins it against the reference's own outputs
(tests/golden, made by tests/golden/make_golden.py from ICON-GPU compiled for
sm_100a) and against mathematics (direct NDFT, adjoint identity)."""
import numpy as np
import pytest

from conftest import load_golden, min_abs_tilt_index, rel_l2
from oracle.oracle import OraclePlan, grid_params

# The reference computes in float with cuFFT; these are relative-L2 bounds of
# oracle vs reference, measured around 2e-7 (stages) and 4e-6 (200 iterations).
TOL_STAGE = 1e-6
TOL_SOLVE = 2e-5


def test_grid_sizes_match_reference_formula():
    # n = 2 * nextpow2(N) for every N (MainCode.cu:66-71).
    for N in list(range(8, 600)) + [1000, 1023, 1024, 1025, 2047, 2048, 4096]:
        th, n, b, bf = grid_params(N)
        p2 = 1
        while p2 < N:
            p2 *= 2
        assert n == 2 * p2, N


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_nufft_vs_direct_ndft(prec):
    tilts = np.arange(-60, 61, 7.5).astype(np.float32)
    p = OraclePlan(40, 24, tilts, prec)
    rng = np.random.default_rng(1)
    img = rng.standard_normal((40, 24))
    assert rel_l2(p.forward(img), p.ndft_forward(img)) < 5e-6
    f = rng.standard_normal(p.M) + 1j * rng.standard_normal(p.M)
    assert rel_l2(p.adjoint(f), p.ndft_adjoint(f)) < 5e-6


@pytest.mark.parametrize("prec,bound", [("f64", 2e-7), ("f32", 4e-7)])
def test_kaiser_bessel_window_vs_direct_ndft(prec, bound):
    """The Kaiser-Bessel mode (half-width 4, no counterpart in the
    reference): non-zero on taps 3..10 of the 14 only, and closer to the
    direct NDFT than the reference's Gaussian of half-width 6."""
    tilts = np.arange(-60, 61, 3).astype(np.float32)
    rng = np.random.default_rng(3)
    for nx, th in ((64, 40), (50, 37), (128, 96)):
        kb = OraclePlan(nx, th, tilts, prec, window="kb4")
        ga = OraclePlan(nx, th, tilts, prec)
        phix, _, phiy, _, cx, cy = kb.windows()
        assert not np.any(phix[:, :3]) and not np.any(phix[:, 11:]), (nx, th)
        assert not np.any(phiy[:, :3]) and not np.any(phiy[:, 11:]), (nx, th)
        assert np.all(cx > 0) and np.all(cy > 0)
        img = rng.standard_normal((nx, th))
        f = rng.standard_normal(kb.M) + 1j * rng.standard_normal(kb.M)
        e_kb = max(rel_l2(kb.forward(img), kb.ndft_forward(img)), rel_l2(kb.adjoint(f), kb.ndft_adjoint(f)))
        e_ga = max(rel_l2(ga.forward(img), ga.ndft_forward(img)), rel_l2(ga.adjoint(f), ga.ndft_adjoint(f)))
        assert e_kb < bound, (nx, th, e_kb)
        assert e_kb < e_ga, (nx, th, e_kb, e_ga)


def test_adjoint_identity_fp64():
    tilts = np.linspace(-58, 61, 17).astype(np.float32)
    p = OraclePlan(33, 21, tilts, "f64")
    rng = np.random.default_rng(2)
    x = rng.standard_normal((33, 21)) + 1j * rng.standard_normal((33, 21))
    y = rng.standard_normal(p.M) + 1j * rng.standard_normal(p.M)
    lhs = np.vdot(y, p.forward(x))
    rhs = np.vdot(p.adjoint(y), x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


@pytest.mark.parametrize("name", ["a", "b", "c", "cli"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_matches_reference_stages(golden, name, prec):
    z = golden[name]
    p = OraclePlan(int(z["nx"]), int(z["thickness"]), z["tilts"], prec)
    assert rel_l2(p.forward(z["img_r"]), z["ref_fwd_r"]) < TOL_STAGE
    assert rel_l2(p.forward(z["img_c"]), z["ref_fwd_c"]) < TOL_STAGE
    assert rel_l2(p.adjoint(z["f"]), z["ref_adj"]) < TOL_STAGE
    for s in range(int(z["S"])):
        assert rel_l2(p.rows_forward(z["rows"][s]), z["ref_b"][s]) < TOL_STAGE
        assert rel_l2(p.rhs(z["rows"][s]), z["ref_Ahwb"][s]) < TOL_STAGE


@pytest.mark.parametrize("name", ["a", "b", "cli"])
def test_oracle_matches_reference_solve(golden, name):
    z = golden[name]
    nx, th = int(z["nx"]), int(z["thickness"])
    p = OraclePlan(nx, th, z["tilts"], "f64")
    om = float(-z["tilts"][min_abs_tilt_index(z["tilts"])])
    lp = OraclePlan(nx, th, None, "f64", line_angle=om)
    a, b, c = [int(v) for v in z["sched"]]
    for s in range(int(z["S"])):
        A = p.rhs(z["rows"][s])
        m = p.solve(A, (a, b, c), int(z["data_type"]), float(z["threshold"]))
        assert rel_l2(m, z["ref_m"][s]) < TOL_SOLVE
        assert rel_l2(p.reproject(lp, m), z["ref_reproj"][s]) < TOL_SOLVE


def test_oracle_matches_reference_solve_200_iterations(golden):
    z = golden["c"]
    p = OraclePlan(int(z["nx"]), int(z["thickness"]), z["tilts"], "f64")
    A = p.rhs(z["rows"][0])
    m = p.solve(A, tuple(int(v) for v in z["sched"]), int(z["data_type"]), float(z["threshold"]))
    assert rel_l2(m, z["ref_m"][0]) < TOL_SOLVE


def test_reference_cli_fixture_consistent_with_harness(golden):
    # The ICON-GPU command-line run and the harness saw the same inputs; the
    # slice files it wrote hold the harness's m, transposed to X fastest
    # (saveMRC_real_inv, saveMRC_real.cu:33-56).
    from feilab_b200 import mrc
    import io, os, tempfile
    z = golden["cli"]
    assert int(z["cli_returncode"]) == 0
    nx, th = int(z["nx"]), int(z["thickness"])
    for s in range(int(z["S"])):
        raw = z[f"cli_mid{s:05d}"].tobytes()
        with tempfile.NamedTemporaryFile(suffix=".mrc", delete=False) as f:
            f.write(raw)
            path = f.name
        try:
            h, d = mrc.read(path)
        finally:
            os.unlink(path)
        assert (int(h["nx"]), int(h["ny"]), int(h["nz"]), int(h["mode"])) == (nx, th, 1, 2)
        np.testing.assert_array_equal(d[0], z["ref_m"][s].T)


@pytest.mark.parametrize("name", ["p1", "p2"])
def test_preprocess_oracle_matches_reference_tool(name):
    # oracle/preprocess.py against the reference ICONPreProcess's own output.
    import oracle.preprocess as pp
    z = load_golden("preprocess")
    st, tilts, th = z[name + "_stack"], z[name + "_tilts"], int(z[name + "_thickness"])
    np.testing.assert_array_equal(pp.preprocess(st), z[name + "_mode_only"])
    got = pp.preprocess(st, tilts, th)
    ref = z[name + "_normalized"]
    assert np.max(np.abs(got - ref)) <= 2e-6 * np.max(np.abs(ref))


MASK_CASES = {
    # name: (thickness, zshift, radius or None (from the FRC files), gauss width or None, masked)
    "frc": (64, 0, None, None, True),
    "radius": (64, 0, 12, 6, True),
    "crop": (40, 5, 15, None, True),
    "nomask": (48, 0, None, None, False),
}


@pytest.mark.parametrize("name", list(MASK_CASES))
def test_mask_oracle_matches_reference_tool(name):
    # oracle/mask.py against the reference ICONMask3's own output volumes.
    import oracle.mask as mk
    z = load_golden("mask")
    th, zs, radius, gw, masked = MASK_CASES[name]
    mids, tilts = z["mids"], z["tilts"]
    n = mids.shape[-1]
    ystart = n // 2 - th // 2 + zs
    ref = z["vol_" + name]
    if not masked:
        np.testing.assert_array_equal(mk.assemble(mids, ystart, th), ref)
        return
    r05, r03, explicit = mk.radius_rates(n, tilts, radius, z["crossV_frc"][:, 1], z["fullRec_frc"][:, 1])
    filt = mk.half_filter(n, tilts, r05, r03, explicit, gw)
    got = mk.apply(mids, filt, ystart, th)
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < 2e-6


@pytest.mark.parametrize("radius", [None, 12, 1000])
def test_mask_radius_rule_matches_oracle(radius):
    # The library's host rule (icon_mask_radius, no GPU needed) against the oracle.
    import oracle.mask as mk
    from feilab_b200 import tools
    z = load_golden("mask")
    cv, fr = z["crossV_frc"][:, 1], z["fullRec_frc"][:, 1]
    n = z["mids"].shape[-1]
    got = tools.mask_radius(n, z["tilts"], radius, cv, fr)
    ref = mk.radius_rates(n, z["tilts"], radius, cv, fr)
    assert got[2] == ref[2]
    assert got[0] == pytest.approx(ref[0], rel=1e-7) and got[1] == pytest.approx(ref[1], rel=1e-7)


def test_frc_matches_reference_crossv_file(golden, tmp_path):
    # icon_frc (host code, no GPU) on the reference ICON-GPU's own
    # GroundTruth and crossV reprojection reproduces its crossV.frc file.
    from feilab_b200 import mrc, tools
    z = golden["cli"]
    imgs = []
    for key in ("cli_GroundTruth_mrc", "cli_crossV_reprojection_mrc"):
        p = tmp_path / (key + ".mrc")
        p.write_bytes(z[key].tobytes())
        imgs.append(mrc.read(str(p))[1][0])
    ref = np.loadtxt(z["cli_crossV_frc"].tobytes().decode().splitlines())
    got = tools.frc(imgs[0], imgs[1], 10)
    assert got.shape == (ref.shape[0],)
    np.testing.assert_allclose(got, ref[:, 1], atol=2e-6)


def test_icon_weights_match_oracle_weights():
    # icon_weights (the weights a plan gives its nodes, also used for the
    # left-out series of icon_loo_sweep) against the oracle's Weight().
    from feilab_b200.icon import weights
    for nx, tilts in [(64, np.linspace(-60, 60, 31)), (50, np.array([-47.0, -20.5, 3.0, 8.0, 52.0])),
                      (128, np.delete(np.arange(-60, 61, 2.0), [0, 30]))]:
        t = np.asarray(tilts, np.float32)
        _, w_o, _ = OraclePlan(nx, 16, t, "f64").geometry()
        assert np.array_equal(weights(nx, t).ravel(), w_o)


def test_reference_and_fp64_oracle_agree_at_production_size():
    # The cfg2 fixture: the reference's 300-iteration result on 16 slices of
    # the 1024x300, 61-tilt workload and the FP64 oracle's on the same rows.
    from conftest import cfg2_fp64
    z = load_golden("cfg2")
    m64 = cfg2_fp64(z)
    for s in range(int(z["S"])):
        assert rel_l2(z["ref_m"][s], m64[s]) < 1e-5
