"""Multi-GPU host logic: one process per GPU, each advancing its own replica of
the workload (independent Sedov instances need no data-path collective).

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
