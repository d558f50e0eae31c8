"""CPU, world size 2 over gloo: the multi-GPU host logic (max over ranks of
the timed region, whole-job rate, member sharding) as bench.py and an
ensemble run use it, with a real process group."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from finitevolx_b200.replicas import max_over_ranks, shard_members, whole_job_rate, world_info


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        r, w = world_info()
        t = max_over_ranks(10.0 + 5.0 * rank)  # rank 1 is the slower one
        members = [(128, 1), (256, 3), (512, 2), (1024, 1), (256, 1), (128, 3)]
        mine = shard_members(members, r, w)
        dist.barrier()
        out[rank] = (r, w, t, whole_job_rate(1000, 4, t, w), mine)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        r, w, t, rate, _ = res[rank]
        assert (r, w) == (rank, world)
        assert t == 15.0  # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 1000 * 4 / 15e-3 / 1e6)
    a, b = res[0][4], res[1][4]
    assert sorted(a + b) == list(range(6)) and not set(a) & set(b)


def test_shard_members_balances_and_covers():
    members = [(n, nl) for n in (128, 256, 512, 1024) for nl in (1, 2, 3)] * 4
    for world in (1, 2, 3, 8):
        parts = [shard_members(members, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(members)))
        loads = [sum(members[i][0] ** 2 * members[i][1] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(n * n * nl for n, nl in members)
    with pytest.raises(ValueError):
        shard_members(members, 2, 2)


def test_single_process_defaults():
    assert world_info() == (0, 1)
    assert max_over_ranks(3.5) == 3.5
