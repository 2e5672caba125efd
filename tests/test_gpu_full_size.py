"""GPU parity at production sizes against the FP64 oracle.

The golden fixtures are small (up to 256 wide); the kernels take other paths
at production sizes: 8-slice groups with unpadded row pairs in the forward
y-pass and two-row strips in the adjoint gather at 1024 x 300, 4-slice
groups and an oversampled width of 4096 at 2048, short rows and odd widths
elsewhere, long y rows (thickness 700 and 1100: oversampled lengths 2048 and
4096, the latter with the y-pass twiddles read from global memory).  These
cases run the operator on the shapes of the 1024x1024x300
workload (61 tilts, -60..60 step 2) and of the mixed-geometry series (widths
up to 2048, thickness 100-400, tilt ranges +-45..70 with 1.5-3 degree steps
and 10% of the tilts dropped), with seeded random inputs, and compare every
stage with the FP64 oracle, a short solve with the float oracle, and the
adjoint identity <A x, y> = <x, A^H y>.
"""
import numpy as np
import pytest

from conftest import rel_l2

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


# (nx, thickness, tilts, slices per call): the 1024x300 workload, then
# mixed-geometry series of the widest, an odd and the thinnest kind.
CASES = {
    "1024x300_61tilts": (1024, 300, _tilts(-60, 60, 2, 0.0, 0), 8),
    "2048x400_drop10": (2048, 400, _tilts(-70, 70, 1.5, 0.1, 1), 4),
    "768x100_drop10": (768, 100, _tilts(-45, 45, 3, 0.1, 2), 8),
    "512x257_drop10": (512, 257, _tilts(-55, 62, 2.5, 0.1, 3), 8),
    # long y rows: n1 = 2048, and n1 = 4096 (twiddles read from global memory)
    "512x700": (512, 700, _tilts(-60, 60, 3, 0.0, 0), 8),
    "256x1100": (256, 1100, _tilts(-60, 60, 4, 0.0, 0), 8),
}


def _t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype=dtype)


@pytest.mark.parametrize("name", list(CASES))
def test_stages_match_fp64_oracle(name):
    from feilab_b200.icon import IconPlan
    from oracle.oracle import OraclePlan
    nx, th, tilts, S = CASES[name]
    p = IconPlan(nx, th, tilts, capacity=S)
    o = OraclePlan(nx, th, tilts, "f64")
    assert (p.M, p.N0, p.N1) == (o.M, o.N0, o.N1)
    rng = np.random.default_rng(11)
    img = rng.standard_normal((S, nx, th)).astype(np.float32)
    f = p.nufft_forward(_t(img)).cpu().numpy()
    fv = (rng.standard_normal((S, p.M)) + 1j * rng.standard_normal((S, p.M))).astype(np.complex64)
    a = p.nufft_adjoint(_t(fv)).cpu().numpy()
    rows = rng.standard_normal((S, len(tilts), nx)).astype(np.float32)
    Ah = p.prepare_rhs(_t(rows)).cpu().numpy()
    for s in (0, S - 1):      # first and last slot of the group
        assert rel_l2(f[s], o.forward(img[s].astype(np.float64))) < TOL_STAGE, (name, s)
        assert rel_l2(a[s], o.adjoint(fv[s].astype(np.complex128))) < TOL_STAGE, (name, s)
        assert rel_l2(Ah[s], o.rhs(rows[s].astype(np.float64))) < TOL_STAGE, (name, s)
    # <A x, y> = <x, A^H y> per slice, in double from the float results
    for s in range(S):
        lhs = np.vdot(fv[s].astype(np.complex128), f[s].astype(np.complex128))
        rhs = np.vdot(a[s].astype(np.complex128), img[s].astype(np.complex128))
        assert abs(lhs - rhs) <= 1e-5 * np.linalg.norm(f[s]) * np.linalg.norm(fv[s]), (name, s)


@pytest.mark.parametrize("name", ["1024x300_61tilts", "2048x400_drop10"])
def test_short_solve_matches_float_oracle(name):
    from feilab_b200.icon import IconPlan
    from oracle.oracle import OraclePlan
    nx, th, tilts, S = CASES[name]
    sched, data_type, thr = (1, 3, 1), 2, 0.0
    p = IconPlan(nx, th, tilts, capacity=S)
    o = OraclePlan(nx, th, tilts, "f32")
    rows = np.random.default_rng(12).standard_normal((S, len(tilts), nx)).astype(np.float32)
    m = p.solve(p.prepare_rhs(_t(rows)), sched, data_type, thr)
    rp = p.reproject(m).cpu().numpy()
    m = m.cpu().numpy()
    lp = OraclePlan(nx, th, None, "f32", line_angle=float(-tilts[p.omit_index]))
    for s in (0, S - 1):
        mo = o.solve(o.rhs(rows[s]), sched, data_type, thr)
        assert rel_l2(m[s], mo) < TOL_SOLVE, (name, s)
        assert rel_l2(rp[s], o.reproject(lp, mo)) < TOL_SOLVE, (name, s)
