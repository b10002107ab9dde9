"""Floating-point operations per zone-update of the reference algorithm, counted
by the oracle's counting build (op_count.cpp) -- test and measurement
infrastructure, not part of the product.

For each workload it runs one warm-up coarse step on the counting build, then
counts the operations of the next coarse step (estdt, the three clean_state
passes, the ghost fill, the per-box hydro of Castro_hydro.cpp and the update)
and divides by the zones.  The workloads:

  sedov128_pert      the perturbed Sedov workload: 128^3 in 64 boxes of 32^3,
                     2 species, outflow
  sedov64            one 64^3 box, 2 species, outflow
  sedov128_pert_64   the perturbed workload's box shape at 64^3 zones (8 boxes
                     of 32^3) ...
  sedov128_pert_1box ... and the same 64^3 domain as one box: the difference is
                     the per-box algorithm's ghost-zone work (ctoprim on
                     grow(box, 4), the trace and Riemann stages on grown boxes)
  reference          the reference problem: 128^3 in 8 boxes of 64^3, 13 species,
                     periodic

"flops" counts add, mul, div, sqrt and transcendental as one each (the
parity build has no fused multiply-adds); compares and sign operations are
listed but not counted.

    python oracle/count_ops.py [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def _package():
    import importlib
    return importlib.import_module("mini-castro_b200")


def count_workload(cfg, table: str, threads: int = 0) -> dict:
    """Operation counts per zone-update of the second coarse step of cfg's first instance."""
    A, Z = cfg["network"]
    O.network_init(A, Z, "count")
    O.eos_init(table, "count")
    inst = cfg["instances"][0]
    nvar = 7 + len(A)
    L, prob = O.level_from_instance(inst, nvar, "count")
    if threads:
        L.set_threads(threads)
    L.coarse_step(1e30)                       # warm-up step (the first step's dt is the initial 0.01 x)
    O.op_counts_reset()
    t0 = time.perf_counter()
    L.coarse_step(1e30)
    wall = time.perf_counter() - t0
    c = O.op_counts()
    nz = 1
    for l, h in zip(inst["dom_lo"], inst["dom_hi"]):
        nz *= h - l + 1
    per = {k: v / nz for k, v in c.items()}
    flops = per["add"] + per["mul"] + per["div"] + per["sqrt"] + per["transcendental"]
    return dict(zones=nz, boxes=len(inst["boxes"]), nspec=len(A),
                per_zone_update={k: round(v, 1) for k, v in per.items()},
                flops_per_zone_update=round(flops, 1), seconds=round(wall, 2))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=None, help="write the counts as JSON here")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    pkg = _package()
    C = pkg.configs
    table = pkg.helm_table.ensure_table()
    runs = {
        "sedov128_pert": C.sedov128_pert(),
        "sedov64": C.sedov64(),
        "sedov128_pert_64": C.sedov128_pert(scale=2, max_box=64),
        "sedov128_pert_1box": C.sedov128_pert(scale=2, max_box=128),
        "reference": C.reference(),
    }
    res = {}
    for name, cfg in runs.items():
        res[name] = count_workload(cfg, table, args.threads)
        print(name, json.dumps(res[name]), flush=True)
    res["_source"] = ("oracle/count_ops.py: the oracle's parity algorithm compiled with every floating-point "
                      "operation counted (oracle/op_count.cpp), one coarse step after a warm-up step, per zone")
    if args.out:
        with open(args.out, "w") as fp:
            json.dump(res, fp, indent=1)
            fp.write("\n")


if __name__ == "__main__":
    main()
