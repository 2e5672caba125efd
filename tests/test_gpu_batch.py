"""Uneven multi-series batches (include/icon_batch.h): many tilt series of
different width, tilt count, thickness and slice count reconstructed
together, each with its own tuned plan, the series' iterations replayed from
CUDA graphs on their own streams.

Every series' result must be what a plan of that series alone gives (the
same kernels and slice groups: bit for bit), whether the series run
concurrently from graphs or one after another, and must match the FP64
oracle's solve of the same rows within the solve tolerance.  The tuning cache
round-trips through its file."""
import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_SOLVE = 1e-4
SCHED = (2, 5, 2)


def _mixed():
    from feilab_b200 import synth
    rng = np.random.default_rng(11)
    specs = [(64, 48, synth.tilt_angles(-60, 60, 4), 5),
             (50, 37, np.sort(rng.uniform(-55, 58, 23)).astype(np.float32), 3),
             (100, 60, np.delete(synth.tilt_angles(-45, 50, 5), [3, 11]), 7),
             (128, 40, synth.tilt_angles(-60, 60, 3), 9)]
    out = []
    for k, (nx, th, tilts, S) in enumerate(specs):
        ph = synth.make_phantom((nx, S, th), 12, 20, seed=50 + k, background=0.1)
        rows = synth.add_noise(synth.project(ph, tilts), 0.3, 50 + k).numpy()
        out.append((nx, th, tilts, S, rows))
    return out


def _plain(nx, th, tilts, S, rows):
    from feilab_b200 import icon
    p = icon.IconPlan(nx, th, tilts, capacity=S)
    p.set_operator("toeplitz")
    m = p.solve(p.prepare_rhs(torch.from_numpy(rows).cuda()), SCHED, 2, 0.0).cpu().numpy()
    B = p.B
    p.close()
    return m, B


def test_mixed_batch_matches_plain_plans_and_fp64_oracle():
    from feilab_b200 import icon
    from oracle.oracle import OraclePlan
    series = _mixed()
    b = icon.IconBatch([(nx, th, t, S) for nx, th, t, S, _ in series], operator="toeplitz")
    rows = [torch.from_numpy(r).pin_memory() for *_, r in series]
    got = b.reconstruct(rows, SCHED, 2, 0.0)
    seq = b.reconstruct(rows, SCHED, 2, 0.0, concurrent=False)
    for k, (nx, th, tilts, S, r) in enumerate(series):
        m = got[k].numpy()
        assert m.shape == (S, nx, th)
        assert np.array_equal(m, seq[k].numpy()), k
        mp, B = _plain(nx, th, tilts, S, r)
        assert b.tuning(k)["group"] == B
        assert np.array_equal(m, mp), k
        o = OraclePlan(nx, th, tilts, "f64")
        for s in range(S):
            mo = o.solve(o.rhs(r[s]), SCHED, 2, 0.0)
            assert rel_l2(m[s], mo) < TOL_SOLVE, (k, s)
    b.close()


def test_batch_chunks_and_tuning_cache(tmp_path):
    # Series longer than their tuned chunk run in several chunks (the last
    # one partial, a graph of its own); the tuning found by timing is written
    # to the cache and read back by the next batch.
    from feilab_b200 import icon
    series = _mixed()[:2]
    shapes = [(nx, th, t, S) for nx, th, t, S, _ in series]
    cache = tmp_path / "tune.txt"
    b = icon.IconBatch(shapes, operator="toeplitz", tune_cache=str(cache), tune=2)
    t0 = [b.tuning(k) for k in range(2)]
    assert all(t["tuned"] == 1 and t["group"] in (1, 2, 4, 8) and t["us_per_slice_iteration"] > 0 for t in t0)
    b.close()
    lines = [ln.split() for ln in cache.read_text().splitlines() if ln.strip()]
    assert len(lines) == 2
    # chunk of 2 slices for both shapes: 5 and 3 slices become chunks 2+2+1 and 2+1
    cache.write_text("".join(f"{nx} {th} {len(t)} {S} 1 2 2 1.0\n" for nx, th, t, S in shapes))
    b = icon.IconBatch(shapes, operator="toeplitz", tune_cache=str(cache), tune=0)
    assert [b.tuning(k)["tuned"] for k in range(2)] == [2, 2]
    assert [b.tuning(k)["chunk"] for k in range(2)] == [2, 2]
    got = b.reconstruct([r for *_, r in series], SCHED, 2, 0.0)
    for k, (nx, th, tilts, S, r) in enumerate(series):
        from feilab_b200 import icon as ic
        p = ic.IconPlan(nx, th, tilts, capacity=2)
        p.set_operator("toeplitz")
        ref = np.concatenate([p.solve(p.prepare_rhs(torch.from_numpy(r[s0:s0 + 2]).cuda()), SCHED, 2, 0.0).cpu().numpy()
                              for s0 in range(0, S, 2)])
        p.close()
        assert np.array_equal(got[k].numpy(), ref), k
    b.close()


def test_nufft_operator_batch():
    # The batch also runs the reference's NUFFT operator (direct launches of
    # its iteration inside the graphs); results equal a plain plan's.
    from feilab_b200 import icon
    series = _mixed()[2:]
    b = icon.IconBatch([(nx, th, t, S) for nx, th, t, S, _ in series], operator="nufft")
    got = b.reconstruct([r for *_, r in series], SCHED, 2, 0.0)
    for k, (nx, th, tilts, S, r) in enumerate(series):
        p = icon.IconPlan(nx, th, tilts, capacity=S)
        m = p.solve(p.prepare_rhs(torch.from_numpy(r).cuda()), SCHED, 2, 0.0).cpu().numpy()
        p.close()
        assert np.array_equal(got[k].numpy(), m), k
    b.close()


def test_plans_of_different_sizes_coexist():
    # A kernel's shared-memory limit is a property of the function, shared by
    # every plan: creating a small plan after a large one must not break the
    # large one's launches (each plan used to set the limit to its own size).
    from feilab_b200 import icon
    rng = np.random.default_rng(5)
    big = icon.IconPlan(2048, 200, np.linspace(-60, 60, 11).astype(np.float32), capacity=4)
    rows = torch.from_numpy(rng.standard_normal((3, 11, 2048)).astype(np.float32)).cuda()
    A = big.prepare_rhs(rows)
    m0 = big.solve(A, (1, 2, 1), 2, 0.0).cpu().numpy()
    small = icon.IconPlan(64, 48, np.linspace(-60, 60, 11).astype(np.float32), capacity=4)
    small.solve(small.prepare_rhs(torch.zeros((2, 11, 64), device="cuda")), (1, 1, 1), 2, 0.0)
    A2 = big.prepare_rhs(rows)
    m1 = big.solve(A2, (1, 2, 1), 2, 0.0).cpu().numpy()
    assert np.array_equal(m0, m1)
    small.close()
    big.close()
