"""Multi-GPU host logic: one process per GPU.  Independent Sedov instances
need no data-path collective, so ranks either advance their own replica of a
workload (weak scaling) or split a workload's instances between them
(``partition_by_zones``, strong scaling).

The only collectives are the timing reductions of the benchmark: the step time
is the slowest rank's, and the whole-job rate counts every rank's zones.
Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of x over all ranks (x itself when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(zones_per_rank: int, steps: int, ms_max: float, world: int) -> float:
    """Zone-updates per second of the whole job under weak scaling."""
    return world * zones_per_rank * steps / (ms_max * 1e-3)


def partition_by_zones(zones: list[int], world: int) -> list[list[int]]:
    """Instance indices per rank, balanced by zone count: the largest remaining
    instance goes to the least-loaded rank (longest-processing-time first).
    Deterministic, so every rank computes the same split without communicating."""
    parts = [[] for _ in range(world)]
    load = [0] * world
    for idx in sorted(range(len(zones)), key=lambda i: (-zones[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(idx)
        load[r] += zones[idx]
    return [sorted(p) for p in parts]
