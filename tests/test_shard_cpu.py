"""Box sharding of one level over ranks on CPU (gloo over 127.0.0.1): the fill
plan, the halo exchange and the dt min-reduction of mini_castro_b200.shard,
with each rank's per-box work done by the oracle's per-routine entry points
(the CUDA kernels need a GPU; tests/test_gpu_shard.py drives them).  Two ranks
advance their halves of the BoxArray in lockstep and every box must equal the
single-rank oracle level bit for bit, dt included -- for an outflow domain of
4^3 boxes and a periodic 13-species one of 8^3 boxes."""
from __future__ import annotations

import ctypes as C
import json
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleKernels:
    """The per-box work of Castro::advance on the oracle (checker side), on
    torch CPU tensors so that the shard module's exchange can send them."""

    CLEAN = ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp")

    def __init__(self, oracle, nvar):
        import torch

        self.O, self.nvar, self.torch = oracle, nvar, torch

    def new(self, lo, hi):
        n = int(np.prod([h - l + 1 for l, h in zip(lo, hi)]))
        return self.torch.zeros(n * self.nvar, dtype=self.torch.float64)

    def clean(self, a, alo, ahi, lo, hi):
        for name in self.CLEAN:
            self.O.call(name, list(lo), list(hi), a.numpy(), list(alo), list(ahi))

    def estdt(self, u, lo, hi, dx) -> float:
        dt = C.c_double(1.79769313486231570e308)
        self.O.lib().oracle_estdt(self.O.ivec(lo), self.O.ivec(hi), u.numpy().ctypes.data_as(C.POINTER(C.c_double)),
                                  self.O.ivec(lo), self.O.ivec(hi), self.O.dvec(dx), C.byref(dt))
        return dt.value

    def hydro_source(self, sb, lo, hi, dom_lo, dom_hi, dx, dt):
        O = self.O
        src = self.new(lo, hi)
        glo, ghi = [l - 4 for l in lo], [h + 4 for h in hi]
        dp = C.POINTER(C.c_double)
        O.lib().oracle_construct_hydro_source_tile(
            O.ivec(lo), O.ivec(hi), sb.numpy().ctypes.data_as(dp), O.ivec(glo), O.ivec(ghi),
            src.numpy().ctypes.data_as(dp), O.ivec(lo), O.ivec(hi), O.ivec(dom_lo), O.ivec(dom_hi), O.dvec(dx),
            C.c_double(dt))
        return src

    def saxpy(self, u, dt, src):
        u.add_(src * dt)

    def gather(self, a, idx):
        return a.view(self.nvar, -1)[:, self.torch.as_tensor(idx)]

    def scatter(self, a, idx, vals):
        a.view(self.nvar, -1)[:, self.torch.as_tensor(idx)] = vals

    def to_host(self, a):
        return a.numpy()

    def from_host(self, x):
        return self.torch.from_numpy(np.array(x, dtype=np.float64))


def _workload(pkg, name):
    if name == "outflow":
        return pkg.configs.sedov128_pert(scale=8, max_box=32)      # 16^3 in 64 boxes of 4^3, 2 species
    return pkg.configs.reference(scale=8, max_box=64)              # 16^3 in eight 8^3 boxes, 13 species, periodic


def _run(pkg, oracle, table, name, rank, world, steps, group=None):
    """This rank's boxes after `steps` sharded coarse steps and the dt sequence,
    with the single-rank oracle level's state and dts beside them."""
    cfg = _workload(pkg, name)
    inst = cfg["instances"][0]
    nv = pkg.configs.nvar(cfg)
    oracle.network_init(*cfg["network"])
    oracle.eos_init(table)
    lev, prob = oracle.level_from_instance(inst, nv)
    lev.set_threads(1)
    G0 = oracle.assemble(lev, inst)
    sl = pkg.shard.ShardedLevel(inst, nv, OracleKernels(oracle, nv), rank, world, group)
    sl.set_state(G0)
    dts = [sl.coarse_step() for _ in range(steps)]
    dto = [lev.coarse_step(-1.0) for _ in range(steps)]
    Go = oracle.assemble(lev, inst)
    out = []
    for b in sl.mine:
        lo, hi = sl.boxes[b]
        sl0 = tuple(slice(l - d, h - d + 1) for l, h, d in zip(lo, hi, inst["dom_lo"]))
        out.append((b, np.array_equal(sl.box_state(b), Go[sl0])))
    return dts, dto, out, sl


def _worker(rank, world, port, out_dir, name):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    from conftest import load_package

    import oracle
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pkg = load_package()
    table = pkg.helm_table.ensure_table()
    dts, dto, out, sl = _run(pkg, oracle, table, name, rank, world, 3)
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fp:
        json.dump({"dts": dts, "dto": dto, "boxes": [[int(b), bool(ok)] for b, ok in out],
                   "sent": [int(sum(pc.dst_idx.size for pc in v)) for v in sl.send.values()]}, fp)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name", ["outflow", "periodic"])
def test_two_ranks_match_single_rank_oracle(tmp_path, pkg, table, name):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path), name), nprocs=2, join=True)
    seen = []
    for r in range(2):
        with open(tmp_path / f"r{r}.txt") as fp:
            res = json.load(fp)
        assert res["dts"] == res["dto"], "dt sequence differs from the single-rank oracle"
        assert res["boxes"] and all(ok for _, ok in res["boxes"]), res["boxes"]
        assert res["sent"] and all(n > 0 for n in res["sent"])     # the halves really exchange halos
        seen += [b for b, _ in res["boxes"]]
    assert sorted(seen) == list(range(len(_workload(pkg, name)["instances"][0]["boxes"])))


def test_fill_plan_covers_every_ghost_zone(pkg):
    """Across all ranks' messages and own copies every Sborder zone of every box
    is filled exactly once, periodic and outflow alike."""
    for cfg in (pkg.configs.batched(scale=8, ninst=0), pkg.configs.reference(scale=8, max_box=32)):
        inst = cfg["instances"][0]
        plan = pkg.shard.FillPlan(inst["boxes"], inst["dom_lo"], inst["dom_hi"], inst["bc"])
        for world in (1, 2, 3):
            owner = pkg.shard.distribute(inst["boxes"], world)
            for b, (lo, hi) in enumerate(plan.boxes):
                n = int(np.prod([h - l + 9 for l, h in zip(lo, hi)]))
                hits = np.zeros(n, dtype=int)
                for src in range(world):
                    for pc in plan.pieces(owner, owner[b], src):
                        if pc.dst_box == b:
                            np.add.at(hits, pc.dst_idx, 1)
                assert (hits == 1).all()


def test_single_rank_is_the_oracle_level(pkg, oracle, table):
    dts, dto, out, _ = _run(pkg, oracle, table, "outflow", 0, 1, 2)
    assert dts == dto and all(ok for _, ok in out)
