"""The tilt-stack input path: rows read on the device straight from a stack
in file order (icon_prepare_rhs_stack, icon_reconstruct_stack), the host
pipeline that streams each batch's results through pinned buffers
(icon_reconstruct_stack_host) and the one-copy upload (icon_stack_upload).

The stack path runs the same kernels on the same values as the row path, so
its results must be bit-identical to icon_prepare_rhs / icon_reconstruct_host
on rows gathered on the host; the reference's own outputs for the whole
command line are checked in test_gpu_cli.py, which runs this path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, TH, NZ, NY = 64, 40, 25, 23
ITERS = (2, 6, 2)


def _tilts(n=NZ):
    return np.linspace(-60, 60, n).astype(np.float32)


def _stack(seed=7, nz=NZ):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nz, NY, NX)).astype(np.float32)


def _rows(stack, y0, S, skip=-1):
    keep = [i for i in range(stack.shape[0]) if i != skip]
    return np.ascontiguousarray(stack[keep][:, y0:y0 + S].transpose(1, 0, 2))


def test_prepare_rhs_stack_equals_rows_path():
    import torch
    from feilab_b200.icon import IconPlan
    st = _stack()
    plan = IconPlan(NX, TH, _tilts(), capacity=16)
    d = torch.from_numpy(st).cuda()
    y0, S = 3, 11
    a = plan.prepare_rhs_stack(d, y0, S)
    b = plan.prepare_rhs(torch.from_numpy(_rows(st, y0, S)).cuda())
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_prepare_rhs_stack_skips_a_section():
    import torch
    from feilab_b200.icon import IconPlan
    st = _stack(seed=8)
    skip = 9
    t = np.delete(_tilts(), skip)
    plan = IconPlan(NX, TH, t, capacity=8)
    d = torch.from_numpy(st).cuda()
    a = plan.prepare_rhs_stack(d, 0, 8, skip_section=skip)
    b = plan.prepare_rhs(torch.from_numpy(_rows(st, 0, 8, skip)).cuda())
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    # skipping the last section and skipping none of a stack one section too
    # long read the same rows
    plan_last = IconPlan(NX, TH, _tilts()[:-1], capacity=8)
    c1 = plan_last.prepare_rhs_stack(d, 0, 8, skip_section=NZ - 1)
    c2 = plan_last.prepare_rhs(torch.from_numpy(_rows(st[:-1], 0, 8)).cuda())
    torch.cuda.synchronize()
    assert torch.equal(c1, c2)


@pytest.mark.parametrize("skip", [-1, 4])
def test_reconstruct_stack_equals_reconstruct_host(skip):
    import torch
    from feilab_b200.icon import IconPlan
    st = _stack(seed=9)
    t = _tilts() if skip < 0 else np.delete(_tilts(), skip)
    plan = IconPlan(NX, TH, t, capacity=4)           # S = 10: three chunks
    y0, S = 5, 10
    m_h, rp_h = plan.reconstruct_host(_rows(st, y0, S, skip), ITERS, 2, 0.0, reproject=True)
    m_d, rp_d = plan.reconstruct_stack(torch.from_numpy(st).cuda(), y0, S, ITERS, 2, 0.0, skip_section=skip,
                                       reproject=True)
    torch.cuda.synchronize()
    assert np.array_equal(m_d.cpu().numpy(), m_h.transpose(0, 2, 1))     # file layout: X fastest
    assert np.array_equal(rp_d.cpu().numpy(), rp_h)


def test_reconstruct_stack_host_streams_batches_in_order():
    import torch
    from feilab_b200.icon import IconPlan, OUT_SLICES, OUT_REPROJECTION
    st = _stack(seed=10)
    plan = IconPlan(NX, TH, _tilts(), capacity=4)
    d = torch.from_numpy(st).cuda()
    y0, S = 2, 10
    m_d, rp_d = plan.reconstruct_stack(d, y0, S, ITERS, 1, 0.03, reproject=True)
    torch.cuda.synchronize()
    got = []

    def sink(s0, count, m, rp):
        got.append((s0, count, m.copy(), rp.copy()))
        return 0

    plan.reconstruct_stack_host(d, y0, S, sink, ITERS, 1, 0.03)
    assert [(g[0], g[1]) for g in got] == [(0, 4), (4, 4), (8, 2)]
    assert np.array_equal(np.concatenate([g[2] for g in got]), m_d.cpu().numpy())
    assert np.array_equal(np.concatenate([g[3] for g in got]), rp_d.cpu().numpy())
    # reprojection only: the slices are not copied
    only = []
    plan.reconstruct_stack_host(d, y0, S, lambda s0, c, m, rp: only.append((m, rp.copy())) or 0, ITERS, 1, 0.03,
                                outputs=OUT_REPROJECTION)
    assert all(m is None for m, _ in only)
    assert np.array_equal(np.concatenate([r for _, r in only]), rp_d.cpu().numpy())
    # slices only
    sl = []
    plan.reconstruct_stack_host(d, y0, S, lambda s0, c, m, rp: sl.append((m.copy(), rp)) or 0, ITERS, 1, 0.03,
                                outputs=OUT_SLICES)
    assert all(r is None for _, r in sl)
    assert np.array_equal(np.concatenate([m for m, _ in sl]), m_d.cpu().numpy())


def test_reconstruct_stack_host_sink_error_stops_the_run():
    import torch
    from feilab_b200.icon import IconPlan, IconError
    st = _stack(seed=11)
    plan = IconPlan(NX, TH, _tilts(), capacity=4)
    d = torch.from_numpy(st).cuda()
    calls = []

    def sink(s0, count, m, rp):
        calls.append(s0)
        return 0 if s0 == 0 else 3

    with pytest.raises(IconError, match="sink"):
        plan.reconstruct_stack_host(d, 0, 12, sink, ITERS, 1, 0.03)
    assert calls == [0, 4]
    # the plan stays usable
    m, _ = plan.reconstruct_stack(d, 0, 4, ITERS, 1, 0.03)
    torch.cuda.synchronize()
    assert np.isfinite(m.cpu().numpy()).all()


def test_stack_upload_packs_the_slice_range():
    import torch
    from feilab_b200.icon import IconPlan, DeviceStack
    st = _stack(seed=12)
    plan = IconPlan(NX, TH, _tilts(), capacity=8)
    y0, S = 6, 9
    ds = DeviceStack(st, 0, y0, S)
    assert ds.shape == (NZ, S, NX)
    ref, rp_ref = plan.reconstruct_stack(torch.from_numpy(st).cuda(), y0, S, ITERS, 2, 0.0, reproject=True)
    torch.cuda.synchronize()
    got = []
    plan.reconstruct_stack_host(ds.ptr, 0, S, lambda s0, c, m, rp: got.append((m.copy(), rp.copy())) or 0,
                                ITERS, 2, 0.0, ny=S)
    ds.close()
    assert np.array_equal(np.concatenate([g[0] for g in got]), ref.cpu().numpy())
    assert np.array_equal(np.concatenate([g[1] for g in got]), rp_ref.cpu().numpy())


def test_stack_arguments_are_checked():
    import torch
    from feilab_b200.icon import IconPlan, IconError
    st = _stack(seed=13)
    plan = IconPlan(NX, TH, _tilts(), capacity=8)
    d = torch.from_numpy(st).cuda()
    with pytest.raises(IconError, match="outside"):
        plan.prepare_rhs_stack(d, NY - 3, 4)
    with pytest.raises(IconError, match="outside"):
        plan.reconstruct_stack(d, -1, 2, ITERS)
    with pytest.raises(IconError, match="skip_section"):
        plan.prepare_rhs_stack(d, 0, 2, skip_section=NZ + 1)
    with pytest.raises(IconError, match="capacity"):
        plan.prepare_rhs_stack(d, 0, 9)
