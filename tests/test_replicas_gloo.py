"""CPU, world size 2 over gloo: the multi-GPU host logic (max over ranks of
the timed region, whole-job rate, member sharding) as bench.py and an
ensemble run use it, with a real process group."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from finitevolx_b200.replicas import (max_over_ranks, shard_members, sharded_ensemble_run, whole_job_rate,
                                      world_info)


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


class _StubEnsemble:
    """Stands in for QGEnsemble on CPU: records which global members it
    holds and how many steps each replay advances them."""

    def __init__(self, idx, log):
        self.idx, self.log, self.launches_per_step = list(idx), log, 7

    def capture(self, n):
        stub = self

        class G:
            def replay(self):
                for i in stub.idx:
                    stub.log[i] = stub.log.get(i, 0) + n
        return G()


def _ens_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        members = [(128, 1), (256, 3), (512, 2), (1024, 1), (256, 1), (128, 3), (512, 1)]
        log = {}
        times = iter([5.0 + rank])  # one timed replay per rank, rank 1 slower
        r = sharded_ensemble_run(members, 3, lambda sub, idx: _StubEnsemble(idx, log),
                                 timer=lambda run: (run(), next(times))[1])
        out[rank] = (r, dict(log))
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_run_covers_every_member_once():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_ens_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    members = [(128, 1), (256, 3), (512, 2), (1024, 1), (256, 1), (128, 3), (512, 1)]
    logs = [res[r][1] for r in range(world)]
    # every member lives on exactly one rank and was stepped by the warm-up
    # replay and the timed replay (2 x 3 steps)
    assert sorted(i for lg in logs for i in lg) == list(range(len(members)))
    assert all(v == 6 for lg in logs for v in lg.values())
    for rank in range(world):
        r = res[rank][0]
        assert r["t_max_ms"] == 6.0 and r["world"] == world
        assert sum(r["members_per_rank"]) == len(members)
        cells = sum(n * n * nl for n, nl in members)
        assert r["cells_per_step"] == cells
        assert r["value"] == pytest.approx(cells * 3 / 6e-3 / 1e6)
        assert sorted(r["mine"]) == sorted(res[rank][1])
