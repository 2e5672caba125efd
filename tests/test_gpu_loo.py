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


def _reduced_plan_reprojection(z, omit, operator="nufft"):
    """The left-out solve of one tilt with a plan built for the series
    without it (the reference's own construction)."""
    import torch
    from feilab_b200.icon import IconPlan
    keep = [k for k in range(len(z["tilts"])) if k != omit]
    S = int(z["S"])
    p = IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"][keep], capacity=S)
    p.set_operator(operator)
    rows = torch.from_numpy(np.ascontiguousarray(z["rows"][:, keep])).cuda()
    m = p.solve(p.prepare_rhs(rows), tuple(int(v) for v in z["sched"]), int(z["data_type"]), float(z["threshold"]))
    return p.reproject(m, float(z["tilts"][omit])).cpu().numpy()


@pytest.mark.parametrize("capacity", [4, 24])
def test_batched_sweep_equals_per_tilt_plans(golden, capacity):
    # One plan over all tilts with per-group weights (omitted tilt at 0)
    # against a plan built without the tilt: the same solve, up to the order
    # in which the step length's double partial sums are combined.
    z = golden["cli"]
    frc, rp, _ = _sweep(z) if capacity == 4 else _sweep_cap(z, capacity)
    nz = len(z["tilts"])
    for omit in (0, nz // 2, nz - 1):
        ref = _reduced_plan_reprojection(z, omit)
        assert rel_l2(rp[omit], ref) < 1e-6, omit


def _sweep_cap(z, capacity):
    from feilab_b200 import tools
    return tools.loo_sweep(z["rows"], int(z["thickness"]), z["tilts"], tuple(int(v) for v in z["sched"]),
                           int(z["data_type"]), float(z["threshold"]), capacity=capacity)


def test_group_weights_set_and_restore(golden):
    import torch
    from feilab_b200.icon import IconPlan, weights
    z = golden["a"]
    S = int(z["S"])
    p = IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    rows = torch.from_numpy(np.ascontiguousarray(z["rows"])).cuda()
    sched = tuple(int(v) for v in z["sched"])
    plain = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    # the plan's own weights given per group change nothing
    w = weights(int(z["nx"]), z["tilts"]).ravel()
    p.set_group_weights(np.stack([w] * ((S + p.B - 1) // p.B)))
    same = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(same, plain)
    # zero weights remove the data term: the solve stays at m = 0
    p.set_group_weights(np.zeros((1, p.M), np.float32))
    zero = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert not np.any(zero[:min(S, p.B)]) and np.array_equal(zero[p.B:], plain[p.B:])
    p.set_group_weights(None)
    back = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(back, plain)


@pytest.mark.parametrize("capacity", [4, 24])
def test_toeplitz_sweep_equals_per_tilt_plans(golden, capacity):
    # The sweep with the Toeplitz operator: groups leaving out the same tilt
    # share one kernel (computed once per distinct weight set of a batch);
    # each left-out solve equals a Toeplitz plan built without the tilt, and
    # stays within the parity bar of the NUFFT sweep.
    from feilab_b200 import tools
    z = golden["cli"]
    args = (z["rows"], int(z["thickness"]), z["tilts"], tuple(int(v) for v in z["sched"]), int(z["data_type"]),
            float(z["threshold"]))
    frc_t, rp_t, _ = tools.loo_sweep(*args, capacity=capacity, operator="toeplitz")
    _, rp_n, _ = tools.loo_sweep(*args, capacity=capacity)
    nz = len(z["tilts"])
    for omit in (0, nz // 2, nz - 1):
        assert rel_l2(rp_t[omit], _reduced_plan_reprojection(z, omit, "toeplitz")) < 1e-6, omit
        assert rel_l2(rp_t[omit], rp_n[omit]) < TOL_SOLVE, omit
    assert np.all(np.isfinite(frc_t))


def test_groups_with_equal_weights_share_a_toeplitz_kernel(golden):
    # Per-group weights where several groups carry the same vector: the
    # Toeplitz solve equals the one with the plan's own weights for those
    # groups, and zero weights still remove the data term.
    import torch
    from feilab_b200.icon import IconPlan, weights
    z = golden["a"]
    rows_np = np.concatenate([z["rows"]] * 4)     # 12 slices: two groups of 8
    S = rows_np.shape[0]
    p = IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    p.set_operator("toeplitz")
    rows = torch.from_numpy(np.ascontiguousarray(rows_np)).cuda()
    sched = tuple(int(v) for v in z["sched"])
    plain = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    G = (S + p.B - 1) // p.B
    w = weights(int(z["nx"]), z["tilts"]).ravel()
    p.set_group_weights(np.stack([w] * G))
    same = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(same, plain)
    assert G >= 2
    if G >= 2:
        ws = np.stack([np.zeros_like(w)] + [w] * (G - 1))
        p.set_group_weights(ws)
        mixed = p.solve(p.prepare_rhs(rows), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
        assert not np.any(mixed[:p.B]) and np.array_equal(mixed[p.B:], plain[p.B:])
    p.close()
