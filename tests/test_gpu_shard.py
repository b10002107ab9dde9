"""The sharded level driver (mini_castro_b200.shard) on the GPU: Castro::advance
over the per-routine C-ABI (clean_state's four Castro_F.H kernels, estdt,
castro_construct_hydro_source_box) with the fill plan's copies, on one rank
here (this machine gives one GPU; the exchange between ranks is covered by
tests/test_shard_cpu.py).  The exact build must equal the oracle level bit for
bit, dt included; the production build within the per-zone tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_harness import RTOL_STEP, assert_match

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
@pytest.mark.parametrize("wl", ["outflow", "periodic"])
def test_sharded_driver_matches_oracle(pkg, table, oracle, wl, exact):
    cfg = (pkg.configs.sedov128_pert(scale=4, max_box=64) if wl == "outflow"
           else pkg.configs.reference(scale=8, max_box=64))          # 32^3 in 8 boxes / 16^3 in 8 boxes, 13 species
    inst = cfg["instances"][0]
    nv = pkg.configs.nvar(cfg)
    oracle.network_init(*cfg["network"])
    oracle.eos_init(table)
    lev, prob = oracle.level_from_instance(inst, nv)
    G0 = oracle.assemble(lev, inst)
    L = pkg.castro.init(*cfg["network"], table, exact=exact)
    sl = pkg.shard.ShardedLevel(inst, nv, pkg.shard.GpuKernels(L, nv), 0, 1)
    sl.set_state(G0)
    for _ in range(3):
        dt = sl.coarse_step()
        dto = lev.coarse_step(-1.0)
        if exact:
            assert dt == dto
        else:
            assert abs(dt / dto - 1) <= 1e-14
    Go = oracle.assemble(lev, inst)
    for b in sl.mine:
        lo, hi = sl.boxes[b]
        s0 = tuple(slice(l - d, h - d + 1) for l, h, d in zip(lo, hi, inst["dom_lo"]))
        assert_match(sl.box_state(b), Go[s0], exact, rtol=10 * RTOL_STEP, what=f"box {b}")
