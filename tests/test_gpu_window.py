"""The Kaiser-Bessel window mode (ICON_WINDOW_KB4) on the GPU.

The reference's window is a Gaussian of half-width 6 with 14 taps per
dimension (nufft_gpu_v8.cu:221-235, :471-476, deapodisation :22-42); that
stays the parity mode.  The Kaiser-Bessel mode uses a window of half-width 4
(8 non-zero taps per dimension), so the y-passes gather 8 x 8 instead of
14 x 14 taps per node.  Checked here against the FP64 oracle built with the
same window (oracle/icon_oracle_core.c, window_taps / deapod), against a
direct non-uniform DFT, through the adjoint identity, in a short solve, and
after the production schedule at the 1024 x 300 / 61-tilt shape against the
Gaussian mode and the FP64 (Gaussian) oracle of tests/golden/cfg2.npz.
"""
import numpy as np
import pytest

from conftest import cfg2_fp64, load_golden, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-5
TOL_SOLVE = 1e-4


def _tilts(lo, hi, step, drop, seed):
    t = np.arange(lo, hi + 1e-3, step).astype(np.float32)
    if drop:
        rng = np.random.default_rng(seed)
        keep = np.sort(rng.choice(len(t), len(t) - int(round(drop * len(t))), replace=False))
        t = t[keep]
    return t


# (nx, thickness, tilts, slices per call): a small case, the 1024x300
# workload (8-slice groups, row pairs, two-row strips) and a wide series
# (4-slice groups at an oversampled width of 4096).
CASES = {
    "64x40_31tilts": (64, 40, _tilts(-60, 60, 4, 0.0, 0), 3),
    "1024x300_61tilts": (1024, 300, _tilts(-60, 60, 2, 0.0, 0), 8),
    "2048x400_drop10": (2048, 400, _tilts(-70, 70, 1.5, 0.1, 1), 4),
    "50x37_drop10": (50, 37, _tilts(-55, 62, 2.5, 0.1, 3), 2),
}


def _t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


@pytest.mark.parametrize("name", list(CASES))
def test_kb_stages_match_fp64_kb_oracle(name):
    from feilab_b200.icon import IconPlan
    from oracle.oracle import OraclePlan
    nx, th, tilts, S = CASES[name]
    p = IconPlan(nx, th, tilts, capacity=S, window="kb4")
    o = OraclePlan(nx, th, tilts, "f64", window="kb4")
    rng = np.random.default_rng(21)
    img = rng.standard_normal((S, nx, th)).astype(np.float32)
    f = p.nufft_forward(_t(img)).cpu().numpy()
    fc = p.nufft_forward(_t(img.astype(np.complex64))).cpu().numpy()
    fv = (rng.standard_normal((S, p.M)) + 1j * rng.standard_normal((S, p.M))).astype(np.complex64)
    a = p.nufft_adjoint(_t(fv)).cpu().numpy()
    rows = rng.standard_normal((S, len(tilts), nx)).astype(np.float32)
    Ah = p.prepare_rhs(_t(rows)).cpu().numpy()
    for s in (0, S - 1):
        fo = o.forward(img[s].astype(np.float64))
        assert rel_l2(f[s], fo) < TOL_STAGE, (name, s)
        assert rel_l2(fc[s], fo) < TOL_STAGE, (name, s)
        assert rel_l2(a[s], o.adjoint(fv[s].astype(np.complex128))) < TOL_STAGE, (name, s)
        assert rel_l2(Ah[s], o.rhs(rows[s].astype(np.float64))) < TOL_STAGE, (name, s)
    for s in range(S):
        lhs = np.vdot(fv[s].astype(np.complex128), f[s].astype(np.complex128))
        rhs = np.vdot(a[s].astype(np.complex128), img[s].astype(np.complex128))
        assert abs(lhs - rhs) <= 1e-5 * np.linalg.norm(f[s]) * np.linalg.norm(fv[s]), (name, s)
    p.close()


def test_kb_is_closer_to_the_direct_ndft_than_the_gaussian():
    """Both windows against the exact non-uniform DFT (the oracle's direct
    NDFT in double): the Kaiser-Bessel window with 8 taps approximates it
    more closely than the Gaussian with 14."""
    from feilab_b200.icon import IconPlan
    from oracle.oracle import OraclePlan
    nx, th, tilts, S = 128, 96, _tilts(-60, 60, 3, 0.0, 0), 2
    rng = np.random.default_rng(22)
    img = rng.standard_normal((S, nx, th)).astype(np.float32)
    fv = (rng.standard_normal((S, nx * len(tilts))) + 1j * rng.standard_normal((S, nx * len(tilts)))).astype(np.complex64)
    d = OraclePlan(nx, th, tilts, "f64")
    err = {}
    for w in ("gauss6", "kb4"):
        p = IconPlan(nx, th, tilts, capacity=S, window=w)
        f = p.nufft_forward(_t(img)).cpu().numpy()
        a = p.nufft_adjoint(_t(fv)).cpu().numpy()
        err[w] = max(max(rel_l2(f[s], d.ndft_forward(img[s].astype(np.float64))) for s in range(S)),
                     max(rel_l2(a[s], d.ndft_adjoint(fv[s].astype(np.complex128))) for s in range(S)))
        p.close()
    assert err["kb4"] < 5e-7, err
    assert err["kb4"] < err["gauss6"], err


@pytest.mark.parametrize("operator", ["nufft", "toeplitz"])
def test_kb_short_solve_matches_fp64_kb_oracle(operator):
    from feilab_b200.icon import IconPlan
    from oracle.oracle import OraclePlan
    nx, th, tilts, S = CASES["1024x300_61tilts"]
    sched, data_type, thr = (1, 3, 1), 2, 0.0
    p = IconPlan(nx, th, tilts, capacity=S, window="kb4")
    p.set_operator(operator)
    o = OraclePlan(nx, th, tilts, "f64", window="kb4")
    rows = np.random.default_rng(23).standard_normal((S, len(tilts), nx)).astype(np.float32)
    m = p.solve(p.prepare_rhs(_t(rows)), sched, data_type, thr)
    rp = p.reproject(m).cpu().numpy()
    m = m.cpu().numpy()
    lp = OraclePlan(nx, th, None, "f64", line_angle=float(-tilts[p.omit_index]), window="kb4")
    for s in (0, S - 1):
        mo = o.solve(o.rhs(rows[s].astype(np.float64)), sched, data_type, thr)
        assert rel_l2(m[s], mo) < TOL_SOLVE, (operator, s)
        assert rel_l2(rp[s], o.reproject(lp, mo)) < TOL_SOLVE, (operator, s)
    p.close()


@pytest.mark.parametrize("operator", ["nufft", "toeplitz"])
def test_kb_production_schedule_against_gaussian(operator):
    """The 16 seeded slices of the 1024x1024x300 workload after the full
    300-iteration schedule: the Kaiser-Bessel mode against the reference's
    result and the FP64 oracle's (both with the Gaussian window), within the
    parity bar of 1e-4 relative L2 per slice and FRC >= 0.99."""
    from feilab_b200 import icon
    from feilab_b200.train_warmstart import frc_mean
    z = load_golden("cfg2")
    S = int(z["S"])
    plan = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S, window="kb4")
    plan.set_operator(operator)
    rows = torch.from_numpy(np.ascontiguousarray(z["rows"])).cuda()
    m = plan.solve(plan.prepare_rhs(rows), tuple(int(v) for v in z["sched"]), int(z["data_type"]),
                   float(z["threshold"])).cpu().numpy()
    plan.close()
    m64 = cfg2_fp64(z)
    for s in range(S):
        assert rel_l2(m[s], z["ref_m"][s]) < TOL_SOLVE, (operator, s)
        assert rel_l2(m[s], m64[s]) < TOL_SOLVE, (operator, s)
    frc = frc_mean(torch.from_numpy(m).double(), torch.from_numpy(m64))
    assert frc.min() >= 0.99


def test_kb_window_rejected_values():
    from feilab_b200 import icon
    import ctypes
    t = np.asarray([-30, 0, 30], np.float32)
    g = icon.Geometry(64, 40, 3, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 2, 0, 7)
    h = ctypes.c_void_p()
    assert icon.lib().icon_plan_create(ctypes.byref(g), ctypes.byref(h)) == 1
    assert b"window" in icon.lib().icon_last_error()
