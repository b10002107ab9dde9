"""The multi-GPU host path on CPU: two ranks over gloo (127.0.0.1), each with
its own replica timing; the benchmark's reductions must take the slowest rank
and count every rank's zones."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from conftest import load_package

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pkg = load_package()
    ms = [12.5, 17.25][rank]                         # rank 1 is the slow one
    m = pkg.replicas.max_over_ranks(ms)
    rate = pkg.replicas.whole_job_rate(1000, 10, m, world)
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fp:
        fp.write(f"{m} {rate}")
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reductions(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        m, rate = map(float, open(tmp_path / f"r{r}.txt").read().split())
        assert m == 17.25
        assert rate == pytest.approx(2 * 1000 * 10 / 17.25e-3)


def test_single_process_is_identity(pkg):
    assert pkg.replicas.max_over_ranks(3.5) == 3.5
    assert pkg.replicas.whole_job_rate(10, 2, 1.0, 1) == pytest.approx(2e4)


def test_partition_by_zones(pkg):
    """Every instance on exactly one rank; loads within one instance of each other
    (longest-processing-time bound); the batched configuration's 33 instances."""
    cfg = pkg.configs.batched()
    zones = [pkg.configs.zones(dict(cfg, instances=[i])) for i in cfg["instances"]]
    for world in (1, 2, 3, 4, 8):
        parts = pkg.replicas.partition_by_zones(zones, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(zones)))
        loads = [sum(zones[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(zones)
    assert pkg.replicas.partition_by_zones(zones, 2) == pkg.replicas.partition_by_zones(list(zones), 2)
