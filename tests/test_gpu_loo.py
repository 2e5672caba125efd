"""Leave-one-out cross validation over every tilt (icon_loo_sweep).

For the tilt the reference itself validates (smallest |angle|), the sweep's
reprojection and FRC must equal the reference ICON-GPU's cross-validation
outputs; for another tilt, the reprojection must equal the FP64 oracle's
solve on the reduced tilt set.  With a relative-step tolerance the sweep
must stop within the schedule.
"""
import numpy as np
import pytest

from conftest import min_abs_tilt_index, rel_l2

pytestmark = pytest.mark.gpu
TOL_SOLVE = 1e-4
TOL_FRC = 2e-3


def _sweep(z, **kw):
    from feilab_b200 import tools
    return tools.loo_sweep(z["rows"], int(z["thickness"]), z["tilts"], tuple(int(v) for v in z["sched"]),
                           int(z["data_type"]), float(z["threshold"]), capacity=4, **kw)


def test_loo_matches_reference_cross_validation(golden, tmp_path):
    from feilab_b200 import mrc
    z = golden["cli"]
    frc, rp, it = _sweep(z)
    omit = min_abs_tilt_index(z["tilts"])
    ref_frc = np.loadtxt(z["cli_crossV_frc"].tobytes().decode().splitlines())[:, 1]
    p = tmp_path / "cv.mrc"
    p.write_bytes(z["cli_crossV_reprojection_mrc"].tobytes())
    ref_rp = mrc.read(str(p))[1][0]
    assert rel_l2(rp[omit], ref_rp) < TOL_SOLVE
    np.testing.assert_allclose(frc[omit], ref_frc, atol=TOL_FRC)
    assert np.all(it == sum(int(v) for v in z["sched"]))


def test_loo_other_tilt_matches_oracle(golden):
    from oracle.oracle import OraclePlan
    z = golden["cli"]
    frc, rp, _ = _sweep(z)
    nx, th = int(z["nx"]), int(z["thickness"])
    omit = 2
    keep = [k for k in range(len(z["tilts"])) if k != omit]
    p = OraclePlan(nx, th, z["tilts"][keep], "f64")
    lp = OraclePlan(nx, th, None, "f64", line_angle=float(-z["tilts"][omit]))
    a, b, c = [int(v) for v in z["sched"]]
    for s in range(int(z["S"])):
        m = p.solve(p.rhs(z["rows"][s][keep]), (a, b, c), int(z["data_type"]), float(z["threshold"]))
        assert rel_l2(rp[omit][s], p.reproject(lp, m)) < TOL_SOLVE
    assert np.all(np.isfinite(frc)) and np.all(np.abs(frc) <= 1.0 + 1e-6)


def test_loo_with_tolerance_stops_within_schedule(golden):
    z = golden["cli"]
    frc_c, _, it_c = _sweep(z)
    frc_t, _, it_t = _sweep(z, tol=0.5)
    a, b, c = [int(v) for v in z["sched"]]
    assert np.all(it_t <= it_c) and np.all(it_t >= a + c)
    assert np.all(np.isfinite(frc_t))
