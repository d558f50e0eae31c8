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
