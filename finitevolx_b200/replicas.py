"""Host logic of the multi-GPU form: one process per GPU, no data-path
collective.

A single QG field does not shard (every stage needs the whole field's DST),
so N GPUs run N independent replicas; ensembles shard by members, each rank
stepping its own members.  The only collectives are timing reductions
(the maximum over ranks) and barriers around the timed region, on whatever
process group the caller set up (NCCL on GPUs; gloo in the CPU tests).
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def world_info() -> tuple[int, int]:
    """(rank, world size) of the default process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(value: float, device=None) -> float:
    """The largest ``value`` over all ranks (every rank gets it)."""
    rank, world = world_info()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, t_max_ms: float, world: int) -> float:
    """Units processed by all ranks per second, in millions, over the slowest
    rank's time (weak scaling: every rank does ``units_per_rank`` per step)."""
    return world * units_per_rank * steps / (t_max_ms * 1e-3) / 1e6


def shard_members(members, rank: int, world: int):
    """Indices of the ensemble members rank ``rank`` steps: members taken
    largest first (cells x layers), each to the rank with the least work so
    far (ties to the lower rank); disjoint over ranks and covering all."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    cost = [int(n) * int(n) * int(nl) for n, nl in members]
    order = sorted(range(len(members)), key=lambda i: (-cost[i], i))
    load = [0] * world
    owner = [0] * len(members)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += cost[i]
    return [i for i in range(len(members)) if owner[i] == rank]


def _cuda_ms(run) -> float:
    """Device milliseconds of run() on the current stream (CUDA events)."""
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    run()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1)


def _reduce_device():
    if dist.is_available() and dist.is_initialized() and dist.get_backend() == "nccl":
        return "cuda"
    return None


def sharded_ensemble_run(members, n_steps: int, factory, timer=None) -> dict:
    """Runs an ensemble sharded by members: this rank builds
    ``factory(sub_members, global_indices)`` (an object with ``capture(n)``
    returning a replayable graph and ``launches_per_step``) from the members
    ``shard_members`` assigns it, replays its graph once untimed, then times
    one replay of ``n_steps`` steps between barriers.  No collective runs
    inside the step; the only ones are the barrier and the reductions of
    the time (maximum over ranks) and of the per-rank member counts.

    Returns the slowest rank's time, the whole-job rate (interior
    layer-cells of all members x steps / s / 1e6), this rank's members and
    the member count of every rank."""
    rank, world = world_info()
    mine = shard_members(members, rank, world)
    sub = [members[i] for i in mine]
    ens = factory(sub, mine) if sub else None
    graph = ens.capture(n_steps) if ens is not None else None
    run = graph.replay if graph is not None else (lambda: None)
    run()  # warm-up replay
    timer = timer or _cuda_ms
    if world > 1:
        dist.barrier()
    ms = timer(run)
    dev = _reduce_device()
    t_max = max_over_ranks(ms, device=dev)
    counts = torch.zeros(world, dtype=torch.float64, device=dev)
    counts[rank] = len(mine)
    if world > 1:
        dist.all_reduce(counts)
        dist.barrier()
    cells = sum(int(n) * int(n) * int(nl) for n, nl in members)
    return {"rank": rank, "world": world, "mine": mine, "t_max_ms": t_max, "rank_ms": ms,
            "cells_per_step": cells, "value": cells * n_steps / (t_max * 1e-3) / 1e6 if t_max > 0 else 0.0,
            "members_per_rank": [int(c) for c in counts.tolist()],
            "launches_per_step": getattr(ens, "launches_per_step", 0) if ens is not None else 0}
