"""Parity at the production configuration (the workload bench.py measures):
16 seeded random slices of the 1024 x 1024 x 300, 61-tilt series with the
full 300-iteration schedule (10,280,10, data type 2, threshold 0), against
the reference's own routines (ref_harness, compiled from the reference
sources) and the FP64 oracle on the same rows (tests/golden/cfg2.npz, made by
tests/golden/make_golden_cfg2.py).  The bar is the north star's: at most
1e-4 relative L2 per slice; FRC of every slice against the FP64 oracle's at
least 0.99.  Both normal operators are checked: the reference's NUFFT pair
and the Toeplitz form."""
import numpy as np
import pytest

from conftest import cfg2_fp64, load_golden, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_SOLVE = 1e-4


@pytest.fixture(scope="module")
def cfg2():
    return load_golden("cfg2")


@pytest.mark.parametrize("operator", ["nufft", "toeplitz"])
def test_production_schedule_matches_reference_and_fp64_oracle(cfg2, operator):
    from feilab_b200 import icon
    from feilab_b200.train_warmstart import frc_mean
    z = cfg2
    S = int(z["S"])
    plan = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
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
