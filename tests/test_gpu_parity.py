"""GPU parity of the CUDA path (through the C ABI) against the reference's own
outputs (tests/golden) and the FP64 oracle.

Tolerances (relative L2): single transforms 1e-5 (FP32 FFTs of different
order than cuFFT; the reference and the oracle differ by ~2e-7), full solves
1e-4 (the bar of ICON-GPU parity: <= 1e-4 per slice).
"""
import numpy as np
import pytest

from conftest import min_abs_tilt_index, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-5
TOL_SOLVE = 1e-4


@pytest.fixture(scope="module")
def icon():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from feilab_b200 import icon as m
    m.lib()
    return m


def _t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


@pytest.mark.parametrize("name", ["a", "b", "c", "cli"])
def test_nufft_pair_matches_reference(icon, golden, name):
    z = golden[name]
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=3)
    img_r = np.repeat(z["img_r"][None], 3, 0)
    img_c = np.repeat(z["img_c"][None], 3, 0)
    fwd_r = p.nufft_forward(_t(img_r, torch.float32)).cpu().numpy()
    fwd_c = p.nufft_forward(_t(img_c, torch.complex64)).cpu().numpy()
    adj = p.nufft_adjoint(_t(np.repeat(z["f"][None], 3, 0), torch.complex64)).cpu().numpy()
    for s in range(3):
        assert rel_l2(fwd_r[s], z["ref_fwd_r"]) < TOL_STAGE
        assert rel_l2(fwd_c[s], z["ref_fwd_c"]) < TOL_STAGE
        assert rel_l2(adj[s], z["ref_adj"]) < TOL_STAGE


@pytest.mark.parametrize("name", ["a", "b", "c", "cli"])
def test_input_stage_matches_reference(icon, golden, name):
    z = golden[name]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    rows = _t(z["rows"], torch.float32)
    b = p.rows_forward(rows).cpu().numpy()
    A = p.prepare_rhs(rows).cpu().numpy()
    for s in range(S):
        assert rel_l2(b[s], z["ref_b"][s]) < TOL_STAGE
        assert rel_l2(A[s], z["ref_Ahwb"][s]) < TOL_STAGE


@pytest.mark.parametrize("name", ["a", "b", "c", "cli"])
def test_solve_and_reprojection_match_reference(icon, golden, name):
    z = golden[name]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    A = p.prepare_rhs(_t(z["rows"], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    m = p.solve(A, sched, int(z["data_type"]), float(z["threshold"]))
    rp = p.reproject(m).cpu().numpy()
    m = m.cpu().numpy()
    assert p.omit_index == min_abs_tilt_index(z["tilts"])
    for s in range(S):
        assert rel_l2(m[s], z["ref_m"][s]) < TOL_SOLVE, (name, s)
        assert rel_l2(rp[s], z["ref_reproj"][s]) < TOL_SOLVE, (name, s)


def test_host_pipeline_matches_device_calls(icon, golden):
    z = golden["a"]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=2)   # forces two chunks
    sched = tuple(int(v) for v in z["sched"])
    m_h, rp_h = p.reconstruct_host(z["rows"], sched, int(z["data_type"]), float(z["threshold"]), reproject=True)
    for s in range(S):
        assert rel_l2(m_h[s], z["ref_m"][s]) < TOL_SOLVE
        assert rel_l2(rp_h[s], z["ref_reproj"][s]) < TOL_SOLVE


def test_odd_sizes_against_fp64_oracle(icon):
    from oracle.oracle import OraclePlan
    rng = np.random.default_rng(5)
    for nx, th, tilts in [(37, 23, np.linspace(-47, 52, 11)), (100, 9, np.linspace(-70, 70, 29)),
                          (8, 8, np.array([-30.0, 0.0, 30.0])), (130, 257, np.linspace(-45, 45, 7))]:
        tilts = np.asarray(tilts, np.float32)
        o = OraclePlan(nx, th, tilts, "f64")
        p = icon.IconPlan(nx, th, tilts, capacity=5)
        S = 5
        img = rng.standard_normal((S, nx, th)).astype(np.float32)
        f = p.nufft_forward(_t(img)).cpu().numpy()
        for s in range(S):
            assert rel_l2(f[s], o.forward(img[s].astype(np.float64))) < TOL_STAGE, (nx, th)
        fv = (rng.standard_normal((S, o.M)) + 1j * rng.standard_normal((S, o.M))).astype(np.complex64)
        a = p.nufft_adjoint(_t(fv)).cpu().numpy()
        for s in range(S):
            assert rel_l2(a[s], o.adjoint(fv[s].astype(np.complex128))) < TOL_STAGE, (nx, th)


def test_batch_independence_and_determinism(icon, golden):
    # Each slice of a batch gives the same result as when solved alone, and a
    # second run gives bit-identical output (no atomics anywhere).
    z = golden["a"]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    A = p.prepare_rhs(_t(z["rows"], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    m1 = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    m2 = p.solve(A, sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
    assert np.array_equal(m1, m2)
    for s in range(S):
        ms = p.solve(A[s:s + 1].contiguous(), sched, int(z["data_type"]), float(z["threshold"])).cpu().numpy()
        assert np.array_equal(ms[0], m1[s])


def test_step_lengths_match_oracle(icon, golden):
    from oracle.oracle import OraclePlan
    z = golden["b"]
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=1)
    o = OraclePlan(int(z["nx"]), int(z["thickness"]), z["tilts"], "f64")
    A = p.prepare_rhs(_t(z["rows"][:1], torch.float32))
    sched = tuple(int(v) for v in z["sched"])
    _, al, rt = p.solve(A, sched, int(z["data_type"]), float(z["threshold"]), history=True)
    _, al_o, rt_o = o.solve(o.rhs(z["rows"][0]), sched, int(z["data_type"]), float(z["threshold"]), history=True)
    assert np.allclose(al[:, 0], al_o, rtol=1e-4)
    assert np.allclose(rt[:, 0], rt_o, rtol=1e-4)


def test_fft_stage_cross_checked_with_cufft(icon):
    # The forward NUFFT written with torch.fft (cuFFT) for the FFT and the
    # oracle's window tables must agree with the library's hand-written FFT.
    from oracle.oracle import OraclePlan
    nx, th = 64, 40
    tilts = np.linspace(-60, 60, 13).astype(np.float32)
    o = OraclePlan(nx, th, tilts, "f32")
    phix, ix, phiy, iy, cx, cy = o.windows()
    rng = np.random.default_rng(9)
    img = rng.standard_normal((nx, th)).astype(np.float32)
    n0, n1 = o.n0, o.n1
    g = torch.zeros((n0, n1), dtype=torch.complex64, device="cuda")
    X = np.arange(nx)
    Y = np.arange(th)
    xs = (X - nx // 2 + n0) % n0
    ys = (Y - th // 2 + n1) % n1
    ck = (cx[:, None] * cy[None, :]).astype(np.float32)
    g[np.ix_(xs, ys)] = _t(img / ck, torch.float32).to(torch.complex64)
    G = torch.fft.fft2(g).cpu().numpy()
    f = np.einsum("jt,js,jts->j", phix, phiy, G[ix[:, :, None], iy[:, None, :]])
    p = icon.IconPlan(nx, th, tilts, capacity=1)
    mine = p.nufft_forward(_t(img[None], torch.float32)).cpu().numpy()[0]
    assert rel_l2(mine, f) < TOL_STAGE


def test_rejects_bad_arguments(icon):
    with pytest.raises(icon.IconError):
        icon.IconPlan(4, 16, [0.0, 10.0])
    with pytest.raises(icon.IconError):
        icon.IconPlan(16, 16, [0.0])
    p = icon.IconPlan(16, 16, [-10.0, 0.0, 10.0], capacity=2)
    with pytest.raises(icon.IconError):
        p.nufft_forward(torch.zeros((3, 16, 16), device="cuda"))
