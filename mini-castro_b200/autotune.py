"""Autotuner for the launch shape of the fused batched step.

The fused kernels of ``csrc/castro_sim.cu`` take their block size (the zones
of one work item) and, per kernel group, the minimum number of resident
blocks per SM handed to the register allocator, from ``csrc/castro_tuned.h``.
This script chooses them by measurement on the GPU it runs on:

    python mini-castro_b200/autotune.py [--workload sedov128_pert] [--steps 20]
                                        [--out mini-castro_b200/csrc/castro_tuned.h]

For each candidate it compiles ``castro_sim.cu`` alone with the candidate's
-D flags, links it with the other objects of the default build into a private
library, and times the batched step of the workload in a fresh process (CUDA
events, after warm-up, best of three runs).  The knobs are searched by
coordinate descent from the current defaults: the block size, then the
register budget of the EOS kernels (front, update), of the final Riemann
kernel, of trace, and of the first two Riemann kernels, then the length of
the zone segment one trace thread walks, whether trace's second pass
(transverse velocities and species) runs as a kernel of its own and its
register budget, which operands riemann2 and riemann3 stage in shared memory, and how many passes of consecutive faces one block of
riemann2 / riemann3 makes.  No knob changes any arithmetic, only register
allocation, the distribution of zones over threads and blocks and the path of
the loads, so every candidate computes the same results; the winner is written as
the header together with the timing table, and ``build.py`` compiles the
library with it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import build as B  # noqa: E402

KNOBS = [
    ("CASTRO_BLOCK", [64, 128, 256]),
    ("CASTRO_MINB_EOS", [0, 2, 3, 4]),
    ("CASTRO_MINB_R3", [0, 2, 3, 4]),
    ("CASTRO_MINB_TRACE", [0, 2, 3, 4]),
    ("CASTRO_MINB_RIEMANN", [0, 3, 4, 5, 6]),
    ("CASTRO_TRACE_SEG", [3, 5, 7, 9]),
    ("CASTRO_TRACE_SPLIT", [0, 1]),
    ("CASTRO_MINB_TRACE2", [0, 6, 8]),
    ("CASTRO_R2_STAGE", [0, 1]),
    ("CASTRO_R3_STAGE", [0, 1]),
    ("CASTRO_R2_ROWS", [1, 2, 4]),
    ("CASTRO_R3_ROWS", [1, 2, 4]),
]
DEFAULTS = {"CASTRO_BLOCK": 128, "CASTRO_MINB_EOS": 4, "CASTRO_MINB_R3": 0, "CASTRO_MINB_TRACE": 3,
            "CASTRO_MINB_RIEMANN": 5, "CASTRO_TRACE_SEG": 5, "CASTRO_R2_STAGE": 1, "CASTRO_R3_STAGE": 1,
            "CASTRO_R2_ROWS": 1, "CASTRO_R3_ROWS": 2,
            "CASTRO_TRACE_SPLIT": 1, "CASTRO_MINB_TRACE2": 0}


def key(cfg: dict) -> str:
    return "_".join(f"{k.replace('CASTRO_', '').replace('_', '').lower()}{cfg[k]}" for k in sorted(cfg))


def compile_variant(cfg: dict, workdir: str) -> str:
    """A private libcastro_b200 with castro_sim.cu built under cfg; returns its path."""
    tag = key(cfg)
    os.makedirs(workdir, exist_ok=True)
    obj = os.path.join(workdir, f"sim_{tag}.o")
    lib = os.path.join(workdir, f"libcastro_{tag}.so")
    if os.path.exists(lib):
        return lib
    defs = [f"-D{k}={v}" for k, v in cfg.items()]
    # the candidate's flags replace a tuned header already present
    cmd = [B.NVCC, *B.ARCH, *B.COMMON, "-DCASTRO_NO_TUNED_HEADER", *defs, "-c",
           os.path.join(B.CSRC, "castro_sim.cu"), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {tag}:\n{r.stderr}")
    others = [os.path.join(B.OBJDIR, f"libcastro_b200_{s.replace('.cu', '.o')}") for s in B.SOURCES
              if s != "castro_sim.cu"]
    r = subprocess.run([B.NVCC, *B.ARCH, "-shared", "-o", lib, obj, *others, "-lcudart"], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed for {tag}:\n{r.stderr}")
    return lib


def time_variant(lib: str, workload: str, steps: int, warmup: int) -> float:
    """ms per batched step of the workload with library lib (fresh process)."""
    env = dict(os.environ, CASTRO_B200_LIB=lib)
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--time-only", "--workload", workload,
                        "--steps", str(steps), "--warmup", str(warmup)], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"timing failed for {lib}:\n{r.stdout}\n{r.stderr}")
    return float(json.loads(r.stdout.strip().splitlines()[-1])["ms_per_step"])


def _time_only(workload: str, steps: int, warmup: int) -> None:
    import importlib.util

    import torch

    spec = importlib.util.spec_from_file_location("mini_castro_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["mini_castro_b200"] = pkg
    spec.loader.exec_module(pkg)
    cfg = pkg.configs.WORKLOADS[workload]()
    L = pkg.castro.init(*cfg["network"], pkg.helm_table.ensure_table())
    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    sim.step(warmup)
    sim.sync()
    st = torch.cuda.ExternalStream(sim.stream())
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sim.step(steps)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        best = ms if best is None else min(best, ms)
    sim.close()
    print(json.dumps({"ms_per_step": best}))


def write_header(path: str, cfg: dict, table: list, workload: str) -> None:
    lines = ["// castro_tuned.h -- launch shape of the fused batched step, chosen by",
             "// mini-castro_b200/autotune.py from timings of the batched step",
             f"// ({workload}) on the GPU it ran on.  Timing table (ms per step):"]
    for c, ms in table:
        lines.append(f"//   {key(c):72s} {ms:8.3f}")
    lines.append("#pragma once")
    lines.append("#ifndef CASTRO_NO_TUNED_HEADER")
    for k in sorted(cfg):
        lines += [f"#ifndef {k}", f"#define {k} {cfg[k]}", "#endif"]
    lines.append("#endif")
    with open(path, "w") as fp:
        fp.write("\n".join(lines) + "\n")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="sedov128_pert")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(B.CSRC, "castro_tuned.h"))
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--time-only", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.time_only:
        _time_only(args.workload, args.steps, args.warmup)
        return
    B.build()
    work = args.workdir or tempfile.mkdtemp(prefix="castro_tune_")
    os.makedirs(work, exist_ok=True)
    best = dict(DEFAULTS)
    table = []
    best_ms = time_variant(compile_variant(best, work), args.workload, args.steps, args.warmup)
    table.append((dict(best), best_ms))
    print(f"start {key(best)}: {best_ms:.3f} ms/step", flush=True)
    for knob, values in KNOBS:
        cands = [dict(best, **{knob: v}) for v in values if v != best[knob]]
        with cf.ThreadPoolExecutor(max_workers=min(len(cands), os.cpu_count() or 1)) as ex:
            libs = list(ex.map(lambda c: compile_variant(c, work), cands))
        for c, lib in zip(cands, libs):
            ms = time_variant(lib, args.workload, args.steps, args.warmup)
            table.append((c, ms))
            print(f"  {key(c)}: {ms:.3f} ms/step", flush=True)
            if ms < best_ms * 0.995:   # a change must win by more than timing noise
                best, best_ms = c, ms
        print(f"{knob}: {best[knob]} -> {best_ms:.3f} ms/step", flush=True)
    write_header(args.out, best, table, args.workload)
    print(json.dumps({"best": best, "ms_per_step": best_ms, "header": args.out}))


if __name__ == "__main__":
    main()
