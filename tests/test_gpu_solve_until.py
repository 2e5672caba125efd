"""icon_solve_until: the ICON solve whose ICON phase stops at a tolerance.

It runs the same iterations as icon_solve (the reference's Iteration3 with
Alpha2) and only measures, at its checks, the relative size of an ICON
update, ||m_new - m_old|| / ||m_new||, to decide when to end the ICON phase.
So with tol = 0 it must give icon_solve's result bit for bit; the step it
reports must equal the one computed from two plain solves one iteration
apart; and a start at the cold-start solution must stop at the first check.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(golden, name="c"):
    from feilab_b200 import icon
    z = golden[name]
    S = int(z["S"])
    p = icon.IconPlan(int(z["nx"]), int(z["thickness"]), z["tilts"], capacity=S)
    A = p.prepare_rhs(torch.from_numpy(np.ascontiguousarray(z["rows"])).cuda())
    sched = tuple(int(v) for v in z["sched"])
    return p, A, sched, int(z["data_type"]), float(z["threshold"])


def test_zero_tolerance_gives_icon_solve(golden):
    p, A, sched, dt, thr = _case(golden, "a")
    m_ref = p.solve(A, sched, dt, thr)
    m, n, step = p.solve_until(A, 0.0, sched, dt, thr, check_every=3)
    torch.cuda.synchronize()
    assert n == sum(sched)
    assert torch.equal(m, m_ref)
    assert np.all(step > 0)


def test_step_matches_two_solves(golden):
    p, A, sched, dt, thr = _case(golden, "c")
    a = sched[0]
    k = 25
    m_prev = p.solve(A, (a, k - 1, 0), dt, thr)
    m_next = p.solve(A, (a, k, 0), dt, thr)
    _, n, step = p.solve_until(A, 0.0, (a, k, 0), dt, thr, check_every=k)
    d = (m_next.double() - m_prev.double()).flatten(1).norm(dim=1)
    ref = (d / m_next.double().flatten(1).norm(dim=1)).cpu().numpy()
    assert n == a + k
    np.testing.assert_allclose(step, ref, rtol=1e-9)


def test_start_at_solution_stops_at_first_check(golden):
    p, A, sched, dt, thr = _case(golden, "c")
    a, b, c = sched
    m_full, n_full, step_full = p.solve_until(A, 0.0, sched, dt, thr, check_every=10)
    tol = 2.0 * float(step_full.max())
    m2, n2, step2 = p.solve_until(A, tol, sched, dt, thr, m0=m_full, check_every=10)
    assert n_full == a + b + c
    assert n2 == a + 10 + c
    assert np.all(step2 <= tol)


def test_bad_arguments(golden):
    from feilab_b200.icon import IconError
    p, A, sched, dt, thr = _case(golden, "a")
    with pytest.raises(IconError):
        p.solve_until(A, -1.0, sched, dt, thr)
    with pytest.raises(IconError):
        p.solve_until(A, 0.1, sched, dt, thr, check_every=0)
