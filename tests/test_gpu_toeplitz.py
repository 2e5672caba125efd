"""The Toeplitz normal operator (icon_plan_set_operator(ICON_OPERATOR_TOEPLITZ)):
A^H W A as a convolution with the exact kernel of the node set.

Against the reference: whole solves on the golden fixtures must stay within
the ICON-GPU parity bar (1e-4 relative L2 per slice; the Toeplitz operator
and the reference's Gaussian-window NUFFT pair differ by the window's error,
~1e-6 relative per application).  Against an exact computation: one
iteration from a random start, with A and A^H the oracle's direct NDFT in
FP64, must agree to float rounding (1e-5), which checks the kernel, the
convolution and the step length's quadratic form on their own.
"""
import numpy as np
import pytest

from conftest import min_abs_tilt_index, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-5
TOL_SOLVE = 1e-4


def _t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


@pytest.mark.parametrize("name", ["a", "b", "c", "cli"])
def test_toeplitz_solve_matches_reference(golden, name):
    from feilab_b200 import icon
    z = golden[name]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    p.set_operator("toeplitz")
    A = p.prepare_rhs(_t(z["rows"], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    m = p.solve(A, sched, int(z["data_type"]), float(z["threshold"]))
    rp = p.reproject(m).cpu().numpy()
    m = m.cpu().numpy()
    assert p.omit_index == min_abs_tilt_index(z["tilts"])
    for s in range(S):
        assert rel_l2(m[s], z["ref_m"][s]) < TOL_SOLVE, (name, s)
        assert rel_l2(rp[s], z["ref_reproj"][s]) < TOL_SOLVE, (name, s)
    p.close()


def _exact_iteration(o, w, m0, Ahwb):
    """One unconstrained iteration with the exact transform (FP64 NDFT):
    rhat = A^H W A m0 - Ahwb, alpha = |rhat|^2 / sum w |A rhat|^2."""
    rh = o.ndft_adjoint(w * o.ndft_forward(m0.astype(np.float64))) - Ahwb
    rtr = float((np.abs(rh) ** 2).sum())
    rtar = float((w * np.abs(o.ndft_forward(rh)) ** 2).sum())
    al = rtr / rtar
    return m0 - al * rh.real, al, rtr


@pytest.mark.parametrize("nx,th,tilts", [
    (37, 23, np.linspace(-47, 52, 11)),
    (64, 48, np.arange(-60, 61, 4)),
    (100, 9, np.linspace(-70, 70, 29)),
    (8, 8, np.array([-30.0, 0.0, 30.0])),
    (48, 70, np.linspace(-60, 60, 15)),      # y-transforms of 192 = 32 x 6 points
    (40, 150, np.linspace(-55, 50, 13)),     # 320 = 32 x 10
    (33, 300, np.linspace(-60, 60, 9)),      # 640 = 32 x 20
])
def test_toeplitz_iteration_matches_exact_transform(nx, th, tilts):
    from feilab_b200 import icon
    from oracle.oracle import OraclePlan
    tilts = np.asarray(tilts, np.float32)
    o = OraclePlan(nx, th, tilts, "f64")
    _, w, _ = o.geometry()
    w = w.astype(np.float64)
    rng = np.random.default_rng(nx + th)
    S = 3
    m0 = rng.standard_normal((S, nx, th)).astype(np.float32)
    Ahwb = (rng.standard_normal((S, nx, th)) + 1j * rng.standard_normal((S, nx, th))).astype(np.complex64)
    p = icon.IconPlan(nx, th, tilts, capacity=S)
    p.set_operator("toeplitz")
    m1, al, rt = p.solve(_t(Ahwb), (1, 0, 0), 2, 0.0, m0=_t(m0), history=True)
    m1 = m1.cpu().numpy()
    for s in range(S):
        me, ale, rte = _exact_iteration(o, w, m0[s], Ahwb[s].astype(np.complex128))
        assert rel_l2(m1[s], me) < TOL_STAGE, (nx, th, s)
        assert abs(al[0, s] - ale) <= TOL_STAGE * abs(ale)
        assert abs(rt[0, s] - rte) <= TOL_STAGE * abs(rte)
    p.close()


def test_toeplitz_batch_independence_and_determinism(golden):
    from feilab_b200 import icon
    z = golden["a"]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    p.set_operator("toeplitz")
    A = p.prepare_rhs(_t(z["rows"], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    m1 = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    m2 = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(m1, m2)
    for s in range(S):
        ms = p.solve(A[s:s + 1].contiguous(), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
        assert np.array_equal(ms[0], m1[s])
    p.close()


def test_toeplitz_switch_back_gives_nufft_result(golden):
    from feilab_b200 import icon
    z = golden["b"]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    A = p.prepare_rhs(_t(z["rows"], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    m_n = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    p.set_operator("toeplitz")
    m_t = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    p.set_operator("nufft")
    m_n2 = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(m_n, m_n2)
    for s in range(S):
        assert rel_l2(m_t[s], m_n[s]) < TOL_SOLVE
    with pytest.raises(KeyError):
        p.set_operator("other")
    p.close()


def test_toeplitz_per_group_weights_equal_separate_plans(golden):
    # Two slice groups with different weight vectors (one tilt's nodes at 0 in
    # the second, as the leave-one-out sweep sets them) give, slice by slice,
    # what a plan with only that group's weights gives.
    from feilab_b200 import icon
    z = golden["c"]
    nx, th, tilts = int(z["nx"]), int(z["thickness"]), z["tilts"]
    p = icon.IconPlan(nx, th, tilts, capacity=16)
    B = p.B
    _, w = p.geometry()
    w2 = w.copy()
    k = 7
    w2[k * nx:(k + 1) * nx] = 0.0
    rows = np.repeat(z["rows"][:1], 2 * B, 0)
    sched = (2, 3, 1)
    p.set_operator("toeplitz")
    A = p.prepare_rhs(_t(rows, torch.float32))
    p.set_group_weights(np.stack([w, w2]))
    m = p.solve(A, sched, 2, 0.0).cpu().numpy()
    p.set_group_weights(np.stack([w2, w]))
    m_sw = p.solve(A, sched, 2, 0.0).cpu().numpy()
    p.set_group_weights(None)
    m_plain = p.solve(A, sched, 2, 0.0).cpu().numpy()
    assert np.array_equal(m[0], m_plain[0])
    assert np.array_equal(m_sw[B], m_plain[B])
    assert np.array_equal(m[B], m_sw[0])
    assert rel_l2(m[B], m[0]) > 1e-3          # the weights matter
    p.close()


@pytest.mark.parametrize("nx,th,ntilt", [
    (1024, 160, 31),    # 8-slice groups, 320-point y transforms (R = 10)
    (512, 257, 21),     # 8-slice groups, 640-point y transforms (R = 20)
    (2048, 200, 21),    # 4-slice groups (oversampled width 4096), 512-point y transforms
    (4096, 100, 11),    # 2-slice groups (oversampled width 8192), 256-point y transforms (R = 8)
    (256, 80, 21),      # 192-point y transforms (R = 6)
    (384, 180, 21),     # 384 (R = 12)
    (1024, 300, 61),    # the production shape: 640 (R = 20)
    (512, 350, 21),     # 768 (R = 24)
    (512, 500, 21),     # 1024 (R = 32)
    (256, 60, 21),      # 128 (R = 4)
])
def test_toeplitz_iteration_matches_nufft_iteration_at_large_shapes(nx, th, ntilt):
    # One iteration from a random start with both normal operators: they are
    # the same operator up to the Gaussian window's error (~1e-6 relative),
    # so m, alpha and ||rhat||^2 agree to 1e-5.  Covers the group sizes and
    # y-transform lengths that the fixtures above do not reach.
    from feilab_b200 import icon
    tilts = np.linspace(-60, 60, ntilt).astype(np.float32)
    p = icon.IconPlan(nx, th, tilts, capacity=8)
    rng = np.random.default_rng(nx + th)
    S = 3
    m0 = rng.standard_normal((S, nx, th)).astype(np.float32)
    Ahwb = (rng.standard_normal((S, nx, th)) + 1j * rng.standard_normal((S, nx, th))).astype(np.complex64)
    res = {}
    for op in ("nufft", "toeplitz"):
        p.set_operator(op)
        m1, al, rt = p.solve(_t(Ahwb), (1, 0, 0), 2, 0.0, m0=_t(m0), history=True)
        res[op] = (m1.cpu().numpy(), al, rt)
    (mn, aln, rtn), (mt, alt, rtt) = res["nufft"], res["toeplitz"]
    for s in range(S):
        assert rel_l2(mt[s], mn[s]) < TOL_STAGE, (nx, th, s)
        assert abs(alt[0, s] - aln[0, s]) <= TOL_STAGE * abs(aln[0, s])
        assert abs(rtt[0, s] - rtn[0, s]) <= TOL_STAGE * abs(rtn[0, s])
    p.close()


@pytest.mark.parametrize("nx,th,S", [(1024, 300, 16), (2048, 400, 8), (512, 257, 16), (64, 40, 2)])
def test_tma_column_staging_is_bit_identical(nx, th, S, monkeypatch):
    # The x-kernels stage their G1, Ahwb, r-hat and m columns by TMA (tensor
    # maps, one thread issuing the loads, bounded mbarrier waits) where a CTA
    # takes two or more slices; ICON_XT_TMA=0 keeps the per-thread cp.async
    # staging.  The arithmetic is the same, so the results are equal bit for
    # bit, for both operators' x-kernels (the NUFFT adjoint's last x-pass and
    # the Toeplitz iteration's), and no wait runs out.
    from feilab_b200 import icon
    tilts = np.linspace(-60, 60, 31).astype(np.float32)
    rng = np.random.default_rng(nx + th)
    rows = rng.standard_normal((S, len(tilts), nx)).astype(np.float32)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("ICON_XT_TMA", flag)
        p = icon.IconPlan(nx, th, tilts, capacity=S)
        A = p.prepare_rhs(_t(rows))
        m_n = p.solve(A, (1, 2, 1), 2, 0.0)          # NUFFT operator: the adjoint x-pass with r-hat
        p.set_operator("toeplitz")
        m_t = p.solve(A, (2, 4, 2), 2, 0.0)
        out[flag] = (A.cpu().numpy(), m_n.cpu().numpy(), m_t.cpu().numpy())
        assert p.device_error() == 0
        p.close()
    for a, b in zip(out["1"], out["0"]):
        assert np.array_equal(a, b)
