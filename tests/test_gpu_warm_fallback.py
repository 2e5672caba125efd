"""The cold-start fallback of the warm-started solve (icon_solve_warm).

The reference always starts from m = 0 (Iteration2.cu:33).  A warm start
from the network is accepted per slice only when the warm result is finite,
its ICON phase reached the relative-step tolerance, and it stays within
max_dist of the cold start's first-INFR-phase iterate; any other slice is
solved again from zero with the full schedule.  Corrupted network outputs
are injected from the host (NaN, a start scaled far off, strong noise):
those slices must come back bit for bit equal to the plain cold solve, and
the accepted ones must agree with it (FRC >= 0.99).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SCHED, DTYPE, THR = (5, 60, 5), 2, 0.0


@pytest.fixture(scope="module")
def case():
    from feilab_b200 import icon, synth
    nx, th, S = 256, 128, 8
    tilts = synth.tilt_angles(-60, 60, 2)
    ph = synth.make_phantom((nx, S, th), 60, seed=41)
    rows = synth.add_noise(synth.project(ph, tilts), 0.5, 41).numpy().astype(np.float32)
    plan = icon.IconPlan(nx, th, tilts, capacity=S)
    plan.set_operator("toeplitz")
    A = plan.prepare_rhs(torch.from_numpy(rows).cuda())
    m_cold = plan.solve(A, SCHED, DTYPE, THR)
    torch.cuda.synchronize()
    yield plan, A, m_cold
    plan.close()


def test_corrupted_starts_are_redone_cold(case):
    from feilab_b200.train_warmstart import frc_mean
    plan, A, m_cold = case
    S = A.shape[0]
    m0 = m_cold.clone()
    m0[2] *= 0.9                                   # a plausible, slightly-off start
    m0[1, 10:20, 5:9] = float("nan")               # a network output with NaNs
    m0[3] *= 1000.0                                # a start scaled far off
    g = torch.Generator(device="cuda").manual_seed(5)
    rms = m_cold[6].pow(2).mean().sqrt()
    m0[6] = 30.0 * rms * torch.randn(m_cold[6].shape, device="cuda", generator=g)   # noise
    m, why, iters = plan.solve_warm(A, m0, tol=0.05, iters=SCHED, data_type=DTYPE, threshold=THR)
    torch.cuda.synchronize()
    assert why[1] == 1, why                        # not finite
    assert why[3] in (2, 3) and why[6] in (2, 3), why
    for s in (0, 2, 4, 5, 7):
        assert why[s] == 0, (s, why)
    for s in (1, 3, 6):                            # redone: the cold result, bit for bit
        assert torch.equal(m[s], m_cold[s]), s
    ok = [0, 2, 4, 5, 7]
    frc = frc_mean(m[ok].double().cpu(), m_cold[ok].double().cpu())
    assert frc.min() >= 0.99, frc
    assert 0 < iters <= sum(SCHED)


def test_good_starts_are_all_accepted(case):
    plan, A, m_cold = case
    m, why, iters = plan.solve_warm(A, m_cold.clone(), tol=0.05, iters=SCHED, data_type=DTYPE, threshold=THR)
    torch.cuda.synchronize()
    assert not why.any(), why
    # The ICON phase stopped at the first check: every slice starts at the
    # cold result, whose steps are already below the tolerance.
    assert iters < sum(SCHED), iters


def test_invalid_acceptance_settings_are_rejected(case):
    from feilab_b200.icon import IconError
    plan, A, m_cold = case
    for kw in ({"tol": 0.0}, {"tol": 0.05, "max_dist": 0.0}, {"tol": 0.05, "check_every": 0}):
        with pytest.raises(IconError):
            plan.solve_warm(A, m_cold.clone(), iters=SCHED, data_type=DTYPE, threshold=THR, **kw)


def test_reconstruct_calls_with_warm_start(case):
    # icon_plan_set_warm_start: the reconstruct calls start each slice from
    # the network's prediction and use icon_solve_warm.  With every network
    # parameter at zero the prediction is m0 = 0, so an accepted slice is the
    # cold solve stopped at the tolerance and a redone one the full cold
    # solve, bit for bit; the counts add up; turning it off restores the
    # plain reconstruction.
    import numpy as np
    from feilab_b200 import icon, synth, warmstart
    plan, A, m_cold = case
    nx, th, S = plan.N0, plan.N1, A.shape[0]
    tilts = synth.tilt_angles(-60, 60, 2)
    ph = synth.make_phantom((nx, S, th), 60, seed=41)
    rows = synth.add_noise(synth.project(ph, tilts), 0.5, 41).numpy().astype(np.float32)
    net = warmstart.Network(plan, capacity=4)
    net.set_params(np.zeros(net.n, np.float32), 1.0)
    tol = 0.05
    warmstart.set_warm_start(plan, net, tol)
    got = plan.reconstruct_host(rows, SCHED, DTYPE, THR)
    acc, redo = warmstart.warm_counts(plan)
    assert acc + redo == S
    m_tol, _, _ = plan.solve_until(A, tol, SCHED, DTYPE, THR)
    m_tol = m_tol.cpu().numpy()
    cold = m_cold.cpu().numpy()
    got = got[0] if isinstance(got, tuple) else got
    got = np.asarray(got)
    for s in range(S):
        assert np.array_equal(got[s], m_tol[s]) or np.array_equal(got[s], cold[s]), s
    warmstart.set_warm_start(plan, None, tol)
    plain = plan.reconstruct_host(rows, SCHED, DTYPE, THR)
    plain = np.asarray(plain[0] if isinstance(plain, tuple) else plain)
    assert np.array_equal(plain, cold)
    net.close()
