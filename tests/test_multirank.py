"""Multi-rank host logic on CPU: two gloo ranks on 127.0.0.1.

Slices are independent solves, so a multi-GPU run shares only geometry; the
tests check that ranks take disjoint slices whose union is the whole job,
that the timing reduction is the max over ranks and the rate the whole-job
rate, and the reference's SM-proportional split (ICONGPU.cu:398-449).
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from feilab_b200 import sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nsteps, per_step, ny, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ys = sharding.rank_slices(rank, world, nsteps, per_step, ny)
        gathered = [None] * world
        dist.all_gather_object(gathered, ys)
        t = sharding.max_over_ranks(1.0 + rank, world)          # rank r "took" 1 + r seconds
        rate = sharding.job_rate(world, per_step, nsteps, t)
        out[rank] = (gathered, t, rate)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ny", [1024, 100000])
def test_two_ranks_shard_disjoint_and_time_is_max(ny):
    world, nsteps, per_step = 2, 3, 128
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), nsteps, per_step, ny, out), nprocs=world,
                           start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    g0, t0, r0 = res[0]
    g1, t1, r1 = res[1]
    assert g0 == g1                                  # every rank saw the same shards
    a, b = g0
    assert len(a) == len(b) == nsteps * per_step
    if ny >= world * nsteps * per_step:
        assert not set(a) & set(b)                   # disjoint slices (weak scaling)
    assert t0 == t1 == 2.0                           # max over ranks
    assert r0 == r1 == pytest.approx(world * per_step * nsteps / 2.0)


def test_single_rank_needs_no_group():
    assert sharding.max_over_ranks(3.5, 1) == 3.5
    assert sharding.rank_slices(0, 1, 2, 4, 5) == [0, 1, 2, 3, 4, 0, 1, 2]


@pytest.mark.parametrize("total,sms", [(1024, [148]), (1024, [148, 148]), (301, [148, 132, 148]),
                                       (7, [148] * 8), (0, [148, 148])])
def test_sm_split_is_a_partition_in_sm_proportion(total, sms):
    parts = sharding.sm_split(total, sms)
    assert len(parts) == len(sms)
    pos = 0
    for (start, count), s in zip(parts, sms):
        assert start == pos and count >= 0
        pos += count
    assert pos == total
    tot = float(sum(sms))
    for (start, count), s in zip(parts[:-1], sms[:-1]):
        assert count == int(s / tot * total)         # floor share, the last device takes the rest


def test_bad_arguments():
    with pytest.raises(ValueError):
        sharding.rank_slices(2, 2, 1, 1, 10)
    with pytest.raises(ValueError):
        sharding.sm_split(10, [])
