"""Scenario sharding for one-process-per-GPU runs.

Power-flow scenarios are independent: each rank keeps a replica of the grid,
its symbolic plan and its Ybus, solves a contiguous slice of the scenario set,
and exchanges nothing inside the Newton loop.  The only collective is an
optional gather of the results at the end (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

from typing import Sequence


def scenario_shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) slice of `total` scenarios for `rank`; slice
    sizes differ by at most one and the slices tile [0, total) in rank order."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("scenario_shard: need 0 <= rank < world")
    if total < 0:
        raise ValueError("scenario_shard: total must be >= 0")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def instance_cost(n_bus: int, batch: int) -> float:
    """Relative cost of solving `batch` scenarios of an n_bus grid: the sparse
    factorization of these meshed grids grows a little faster than linearly."""
    return float(batch) * float(n_bus) ** 1.2


def balance_instances(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assign instances (e.g. grids of an uneven multi-grid batch) to ranks by
    longest-processing-time-first; ties go to the lower rank, so every rank
    computes the same assignment without communicating."""
    if world <= 0:
        raise ValueError("balance_instances: world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def gather_rows(local, world: int):
    """All-gather per-rank row blocks (torch tensors, first dim may differ by
    rank) and concatenate them in rank order.  Uses the default process group."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return local
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    rows = [int(s.item()) for s in sizes]
    mx = max(rows)
    pad = torch.zeros((mx,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad)
    return torch.cat([b[:r] for b, r in zip(bufs, rows)], dim=0)
