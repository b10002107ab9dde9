"""Benchmark: zone-updates/s of the CTU hydro advance on B200.

Default workload (the configuration the metric is quoted on): a 128^3 Sedov
blast split into 64 boxes of 32^3, two species, outflow boundaries, ambient
density perturbed by 1e-3 x a seeded Gaussian field, 50 coarse steps
(warm-up + timed).  One "step" is one Amr coarse step of the whole level
(computeNewDt + Castro::advance + post_timestep) over all 2,097,152 zones.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* ``value``: batched fused path, state resident in HBM, device-timed with CUDA
  events on the simulation's stream, max over ranks, summed over ranks.
* ``e2e``: the same metric through the public C-ABI call castro_sim_run_host:
  host->device copy of the state, K steps, device->host copy of the result.
* ``plain_per_box``: the reference's launch structure (one launch per routine
  per box) on the same workload.
* ``roofline``: the dominant fused kernel, from per-kernel CUDA events.
* ``cpu_baseline`` / ``--impl reference``: the C oracle (the reference cannot
  be compiled in this image) on the host cores, OpenMP over MFIter-style tiles.
Multi-GPU (torchrun): every rank advances its own replica of the workload
(independent instances, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "mini-castro_b200")
METRIC = "zone-updates/s on 1 B200: batched vs plain per-box; adjoint/forward time"


def load_package():
    spec = importlib.util.spec_from_file_location("mini_castro_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mini_castro_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            p = json.load(fp)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of this process's GPU, read
    through NVML every 10 ms on a background thread while the timed region
    runs (the GPU is found by its PCI bus id, so CUDA_VISIBLE_DEVICES does not
    matter).  Readings only: no setting of the GPU is touched.  The samples are
    also written as CSV to the file named by $CASTRO_CLOCKS_CSV, if set."""

    PERIOD_S = 0.01

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.rows = []
        self.err = None
        self.path = os.environ.get("CASTRO_CLOCKS_CSV")

    def _handle(self):
        import pynvml as nv
        import torch

        nv.nvmlInit()
        pr = torch.cuda.get_device_properties(self.cuda_index)
        try:
            return nv.nvmlDeviceGetHandleByPciBusId(f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _loop(self):
        import pynvml as nv

        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.rows.append((time.time(), sm, pw, [n for n, b in bits.items() if r & b]))
            except Exception as e:          # keep the first error for the summary
                self.err = self.err or repr(e)
            self.stop.wait(self.PERIOD_S)

    def __enter__(self):
        import threading

        import pynvml as nv

        self.stop = threading.Event()
        self.t = None
        try:
            self.h = self._handle()
            self.sm_max = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
        except Exception as e:
            self.err = repr(e)
        return self

    def __exit__(self, *a):
        if self.t:
            self.stop.set()
            self.t.join(timeout=5)
        if not self.path:
            return
        try:
            os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
            with open(self.path, "w") as fp:
                fp.write("unix_time,sm_mhz,sm_max_mhz,power_w,reasons\n")
                for t, sm, pw, rs in self.rows:
                    fp.write(f"{t:.3f},{sm},{getattr(self, 'sm_max', '')},{pw:.1f},{'|'.join(rs)}\n")
        except OSError:
            pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "error": self.err}
        sm = sorted(r[1] for r in self.rows)
        reasons = sorted({n for r in self.rows for n in r[3]})
        return {"sm_mhz": float(sm[len(sm) // 2]), "sm_max_mhz": float(self.sm_max), "reasons": reasons,
                "samples": len(self.rows), "sm_mhz_min": float(sm[0]), "source": "NVML, 10 ms"}


def kernel_bytes(cfg, nspec):
    """Compulsory HBM bytes of one launch of each fused kernel (every array the
    kernel reads or writes touched once).  front and update walk the boxes of
    the BoxArray; ghost fills each instance's domain halo; prep, trace and the
    three Riemann kernels walk each instance's domain as one region."""
    NV, NQF, NQS, NTF = 7 + nspec, 8 + nspec, 6 + nspec, 7 + nspec
    tot = dict(front=0, ghost=0, trace=0, trace2=0, riemann1=0, riemann2=0, riemann3=0, riemann23=0, update=0)

    def regions(n):
        v = n[0] * n[1] * n[2]
        g1 = (n[0] + 2) * (n[1] + 2) * (n[2] + 2)
        g4 = (n[0] + 8) * (n[1] + 8) * (n[2] + 8)

        def tbx(a, b):
            m = list(n)
            m[a] += 1
            for c in range(3):
                if c != a and c != b:
                    m[c] += 2
            return m[0] * m[1] * m[2]

        def ebx(d):
            m = list(n)
            m[d] += 1
            return m[0] * m[1] * m[2]

        tdd = sum(tbx(d, d) for d in range(3))
        tab = sum(tbx(a, b) for a in range(3) for b in range(3) if a != b)
        eb = sum(ebx(d) for d in range(3))
        return v, g1, g4, tdd, tab, eb

    for inst in cfg["instances"]:
        nd = [h - l + 1 for l, h in zip(inst["dom_lo"], inst["dom_hi"])]
        vd, g1d, g4d, tdd, tab, eb = regions(nd)
        tot["ghost"] += 8 * ((g4d - vd) * NQF * 2 + (g1d - vd) * NV * 2)
        # trace pass 1: rho, u_D, p, rhoe, gamma_1, c and flatn -> 4 face-state components on each side;
        # pass 2 (trace2): the two transverse velocities and the species (+ u_D, flatn) -> the rest
        tot["trace"] += 8 * (g4d * 6 + tdd * 2 * 4 + g1d)
        tot["trace2"] += 8 * (g4d * (3 + nspec) + tdd * 2 * (2 + nspec) + g1d)
        tot["riemann1"] += 8 * (tdd * 2 * NQS + g4d * 2 + tdd * NTF)
        # one thread per face of tbx[a][a] reads its two trace states once for both cross fluxes
        tot["riemann2"] += 8 * (tdd * 2 * NQS + tdd * NTF + g4d * 2 + tab * NTF)
        tot["riemann3"] += 8 * (eb * 2 * NQS + tab * NTF + g1d * NV + g1d + g4d * 2 + eb * (NV + 1))
        # riemann2 + riemann3 per column tile: the cross-flux records stay in shared memory
        tot["riemann23"] += 8 * (tdd * 2 * NQS + tdd * NTF + g4d * 2 + g1d * NV + g1d + eb * (NV + 1))
        tot["update"] += 8 * eb * (NV + 1)   # every final-flux record of the domain read once
        for lo, hi in inst["boxes"]:
            v = regions([h - l + 1 for l, h in zip(lo, hi)])[0]
            tot["front"] += 8 * (v * NV * 2 + v * NV + v * NQF)
            tot["update"] += 8 * v * NV * 2
    return tot


def algorithmic_bytes_per_zone(nspec: int) -> int:
    """HBM bytes one zone-update must move: the conserved state read once and
    written once, 2 x NVAR x 8 B (144 B for 2 species, 320 B for 13)."""
    return 2 * (7 + nspec) * 8


def fp64_block(flops: float, ms: float, peak: float) -> dict:
    ach = flops / (ms * 1e-3) / 1e12
    return {"achieved": ach, "frac": ach / peak if peak else None}


def path_roofline(zones, ms_per_step, bpz, hbm, flops_per_zone, fp64_peak, ref_flops=None) -> dict:
    """Step-level roofline of a whole path: algorithmic bytes and the counted
    FP64 work of the batched step per zone-update, over the path's step time
    (and, when given, the reference algorithm's counted operations)."""
    gbs = zones * bpz / (ms_per_step * 1e-3) / 1e9
    out = {"hbm": {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                   "algorithmic_bytes_per_zone_update": bpz}}
    if flops_per_zone:
        out["fp64"] = dict(fp64_block(zones * flops_per_zone, ms_per_step, fp64_peak), peak=fp64_peak,
                           unit="TFLOP/s", flops_per_zone_update=flops_per_zone)
    if ref_flops:
        out["fp64_reference_algorithm"] = dict(fp64_block(zones * ref_flops, ms_per_step, fp64_peak),
                                               peak=fp64_peak, unit="TFLOP/s", flops_per_zone_update=ref_flops)
    return out


def reference_algorithm_ops(workload: str):
    """The reference algorithm's floating-point operations per zone-update of a
    workload, as the oracle's counting build measured them (oracle/count_ops.py)."""
    path = os.path.join(ROOT, "profiles", "fp64_ops_reference_algorithm.json")
    if not os.path.exists(path):
        return None
    with open(path) as fp:
        return json.load(fp).get(workload)


def run_b200(args, pkg, rank, world):
    import numpy as np
    import torch

    if args.workload == "sedov128_pert" and args.scale > 1:
        # fewer boxes of the same 32^3 shape, so per-zone traffic stays comparable
        cfg = pkg.configs.sedov128_pert(scale=args.scale, max_box=32 * args.scale)
    else:
        cfg = pkg.configs.WORKLOADS[args.workload](scale=args.scale)
    A, Z = cfg["network"]
    nspec = len(A)
    table = pkg.helm_table.ensure_table()
    L = pkg.castro.init(A, Z, table)
    zones = pkg.configs.zones(cfg)
    dev = torch.cuda.current_device()

    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    init_state = sim.download()                      # host copy for the e2e leg
    stream = torch.cuda.ExternalStream(sim.stream())
    for _ in range(args.warmup):
        sim.step(1)
    sim.sync()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        sim.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
    ms = pkg.replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    launches = sim.launches_per_step() * args.steps
    failures = sim.eos_failures()

    # per-kernel breakdown (one extra non-graph step) for the roofline
    prof = sim.profile_step()
    sim.close()
    l2_window = table_window_effect(pkg, L, cfg) if rank == 0 and args.plain_steps > 0 else None

    # e2e through the public C-ABI call with host buffers
    sim2 = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    host_in = torch.from_numpy(init_state).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    sim2.L.castro_sim_run_host(sim2.h, host_in.data_ptr(), 1, host_out.data_ptr())   # instantiates the step graph
    t0 = time.perf_counter()
    rc = sim2.L.castro_sim_run_host(sim2.h, host_in.data_ptr(), args.steps, host_out.data_ptr())
    t_e2e = time.perf_counter() - t0
    pkg.castro.check(L, f"castro_sim_run_host rc={rc}")
    sim2.close()
    t_e2e = pkg.replicas.max_over_ranks(t_e2e, device="cuda")

    # the per-box paths, a few steps: the reference's launch structure through the per-routine
    # entry points (plain), and the same host sequence with each box's hydro source from the
    # coarse drop-in castro_construct_hydro_source_box (plain_box)
    def time_per_box(mode):
        sim3 = pkg.make_sim(L, cfg, mode)
        sim3.init_data()
        sim3.step(2)
        sim3.sync()
        s3 = torch.cuda.ExternalStream(sim3.stream())
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(s3)
        sim3.step(args.plain_steps)
        p1.record(s3)
        p1.synchronize()
        pms = p0.elapsed_time(p1)
        out = {"value": zones * args.plain_steps / (pms * 1e-3), "ms_per_step": pms / args.plain_steps,
               "steps": args.plain_steps, "launches_per_step": sim3.launches_per_step()}
        sim3.close()
        return out

    plain = plain_box = persistent = None
    if rank == 0 and args.plain_steps > 0:
        plain = time_per_box(pkg.castro.MODE_PLAIN)
        plain_box = time_per_box(pkg.castro.MODE_PLAIN_BOX)
    if rank == 0 and args.persistent_steps > 0:
        persistent = time_mode(pkg, L, cfg, pkg.castro.MODE_PERSISTENT, args.persistent_steps, zones)
    column_tiles = None
    if rank == 0 and args.column_tile_steps > 0 and nspec == 2:
        # riemann2 + riemann3 as one column-tile kernel with the cross fluxes in shared memory (opt-in)
        L.castro_set_column_tiles(1)
        try:
            column_tiles = time_mode(pkg, L, cfg, pkg.castro.MODE_BATCHED, args.column_tile_steps, zones)
            sim_ct = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
            sim_ct.init_data()
            sim_ct.step(2)
            column_tiles["kernel_ms"] = sim_ct.profile_step()
            sim_ct.close()
        finally:
            L.castro_set_column_tiles(0)

    batched_cfg = None
    if args.batched_steps > 0:      # every rank: the instances are split over the ranks
        batched_cfg = run_batched_config(pkg, L, args, rank, world)
    large_cfg = None
    if rank == 0 and args.large_steps > 0:
        big = pkg.configs.large()
        large_cfg = {"workload": "large: 384^3 Sedov in an uneven BoxArray of 32^3..64^3 boxes, perturbed density, "
                                 "2 species (the 100-step run timed over its first steps)",
                     "zones": pkg.configs.zones(big), "boxes": len(big["instances"][0]["boxes"]),
                     "batched": time_mode(pkg, L, big, pkg.castro.MODE_BATCHED, args.large_steps,
                                          pkg.configs.zones(big))}
    fd_leg = None
    if rank == 0 and args.fd_table_steps > 0 and nspec == 2:
        # The Fermi-Dirac electron-positron table: the configurations' 1e49-1e51 erg blasts reach ~1e16 K,
        # three decades above the table, where the pair plasma's free energy (~T^4) does not extrapolate; so
        # the headline geometry with a 1e24 erg blast (a pair plasma at ~5e9 K), timed on both tables
        fcfg = fd_workload(pkg)
        fd_path = pkg.helm_fd.ensure_table()
        fd_leg = {"workload": "sedov128_pert geometry and perturbation, blast energy 1e24 erg (inside the table)",
                  "table": "Fermi-Dirac electron-positron gas in pair equilibrium (helm_fd.py)",
                  "helm_table_sha256": pkg.helm_table.sha256(fd_path),
                  "analytic_table": time_mode(pkg, L, fcfg, pkg.castro.MODE_BATCHED, args.fd_table_steps, zones)}
        L.castro_eos_init_path(fd_path.encode())
        pkg.castro.check(L, "eos_init (Fermi-Dirac table)")
        fd_leg["fd_table"] = time_mode(pkg, L, fcfg, pkg.castro.MODE_BATCHED, args.fd_table_steps, zones)
        L.castro_eos_init_path(table.encode())
        pkg.castro.check(L, "eos_init")
    adjoint_cfg = None
    if rank == 0 and args.adjoint_reps > 0:
        adjoint_cfg = run_adjoint_config(pkg, args)
    if rank == 0 and args.large_adjoint > 0:
        large_cfg = dict(large_cfg or {}, adjoint=run_large_adjoint(pkg))

    value = pkg.replicas.whole_job_rate(zones, args.steps, ms, world)
    hbm, peak_kind = peaks()
    fp64_peak = float(L.castro_measure_fp64_tflops())
    step_ms = ms / args.steps
    # algorithmic bytes per zone-update: the state read once and written once, 2 x NVAR x 8 B
    alg_bpz = algorithmic_bytes_per_zone(nspec)
    kb = kernel_bytes(cfg, nspec)
    dom = max((k for k in prof if k in kb), key=lambda k: prof[k])
    fpz = {}
    fpz_path = os.path.join(ROOT, "profiles", "fp64_flops_per_zone.json")
    if os.path.exists(fpz_path):
        with open(fpz_path) as fp:
            fpz = json.load(fp)
    flops_per_zone = fpz.get(args.workload)
    per_kernel = fpz.get(args.workload + "_per_kernel", {})
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    if os.path.exists(tr_path):
        with open(tr_path) as fp:
            traffic = json.load(fp).get(args.workload, {}).get(dom)
    roof_fp64 = None
    if flops_per_zone:
        roof_fp64 = {"bound": "fp64", "kernel": dom, "unit": "TFLOP/s", "peak": fp64_peak,
                     "peak_kind": "measured (DFMA-chain probe kernel, this run)",
                     "flops_per_zone_update": flops_per_zone,
                     "step": fp64_block(zones * flops_per_zone, step_ms, fp64_peak)}
        if per_kernel.get(dom):
            roof_fp64.update(fp64_block(zones * per_kernel[dom], prof[dom], fp64_peak))
            roof_fp64["kernel_flops_per_zone_update"] = per_kernel[dom]
    ref_ops = reference_algorithm_ops(args.workload)
    ref_flops = ref_ops["flops_per_zone_update"] if ref_ops else None
    if roof_fp64 is not None and ref_ops:
        # the survey's FP64 fraction: zone-updates/s x the reference algorithm's counted operations
        # (add, mul, div, sqrt, transcendental as one each) / the measured FP64 peak.  This build
        # executes fewer (flops_per_zone_update, counted by ncu with an FMA as two): no per-box
        # ghost-zone recompute, energy-only Newton evaluations, the table cell by a settled log2.
        roof_fp64["reference_algorithm"] = dict(
            fp64_block(zones * ref_flops, step_ms, fp64_peak), flops_per_zone_update=ref_flops,
            ops_per_zone_update=ref_ops["per_zone_update"],
            source="oracle/count_ops.py: the oracle's parity algorithm with every floating-point operation counted")
    alg = zones * alg_bpz
    roof = {"bound": "hbm", "kernel": dom, "unit": "GB/s", "peak": hbm, "peak_kind": peak_kind,
            "algorithmic_bytes_per_zone_update": alg_bpz, "algorithmic_bytes_per_launch": alg,
            "achieved": alg / (prof[dom] * 1e-3) / 1e9, "frac": alg / (prof[dom] * 1e-3) / 1e9 / hbm,
            "traffic": traffic,
            "step": {"achieved": alg / (step_ms * 1e-3) / 1e9, "frac": alg / (step_ms * 1e-3) / 1e9 / hbm},
            "kernel_compulsory": {
                "bytes_per_launch": kb[dom], "achieved": kb[dom] / (prof[dom] * 1e-3) / 1e9,
                "frac": kb[dom] / (prof[dom] * 1e-3) / 1e9 / hbm,
                "traffic_over_compulsory": traffic / kb[dom] if traffic else None,
                "traffic_over_algorithmic": traffic / alg if traffic else None,
                "note": "bytes of every array the kernel itself reads or writes, touched once (its "
                        "intermediates included): how well it streams what the design keeps in HBM"}}
    for leg in (plain, plain_box):
        if leg:
            leg["roofline"] = path_roofline(zones, leg["ms_per_step"], alg_bpz, hbm, flops_per_zone, fp64_peak,
                                            ref_flops)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "zone-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: Sedov blast, seeded Gaussian density perturbation (numpy PCG64), generated Helmholtz table",
        "config": {"workload": workload_text(args),
                   "zones": zones, "boxes": sum(len(i["boxes"]) for i in cfg["instances"]),
                   "path": "batched fused kernels, one CUDA graph per step",
                   "l2": "no flush: the state plus the per-step intermediates (~1.7 KB/zone) exceed the 126 MB L2",
                   "parallelism": f"replicas x{world}",
                   "helm_table_sha256": pkg.helm_table.sha256(table)},
        "e2e": {"value": pkg.replicas.whole_job_rate(zones, args.steps, t_e2e * 1e3, world), "unit": "zone-updates/s",
                "h2d_bytes_per_step": host_in.numel() * 8 / args.steps,
                "d2h_bytes_per_step": host_out.numel() * 8 / args.steps,
                "call": "castro_sim_run_host (upload state, K steps, download state)"},
        "gpu_launches": launches,
        "kernel_ms": prof,
        "roofline_fp64": roof_fp64,
        "roofline": roof,
        "plain_per_box": plain,
        "plain_box_drop_in": plain_box,
        "persistent": persistent,
        "column_tiles": column_tiles,
        "batched_config": batched_cfg,
        "fd_table": fd_leg,
        "large_config": large_cfg,
        "adjoint_config": adjoint_cfg,
        "adjoint_forward_ratio": adjoint_cfg["adjoint_forward_ratio"] if adjoint_cfg else None,
        "eos_newton_failures": failures,
        "table_l2_window": l2_window,
        "clocks": clk.summary(),
    }
    return line


def fd_workload(pkg):
    """The headline workload's geometry, boxes and density perturbation with a 1e24 erg blast, whose
    states stay inside the Helmholtz table's 1e3..1e13 K."""
    base = pkg.configs.sedov128_pert()
    inst = base["instances"][0]
    return dict(base, instances=[dict(inst, problem=dict(inst["problem"], exp_energy=1e24))])


def time_mode(pkg, L, cfg, mode, steps, zones):
    """zone-updates/s of one sim mode on a workload, device-timed on the sim's stream
    after two untimed steps (the persistent mode: the batched step as one cooperative
    launch per step over device work queues)."""
    import torch

    sim = pkg.make_sim(L, cfg, mode)
    sim.init_data()
    sim.step(2)
    sim.sync()
    st = torch.cuda.ExternalStream(sim.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.step(steps)
    e1.record(st)
    e1.synchronize()
    sim.sync()
    ms = e0.elapsed_time(e1)
    out = {"value": zones * steps / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps,
           "launches_per_step": sim.launches_per_step()}
    sim.close()
    return out


def table_window_effect(pkg, L, cfg, reps=3):
    """The EOS kernels (front, update: every EOS solve of the step) with and without
    the EOS table's persisting L2 access-policy window: median of `reps` profiled steps each."""
    import numpy as np

    out = {}
    for on in (0, 1):
        L.castro_set_table_l2_window(on)
        sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
        sim.init_data()
        sim.step(2)
        runs = [sim.profile_step() for _ in range(reps)]
        sim.close()
        out["on" if on else "off"] = {k: float(np.median([r[k] for r in runs])) for k in ("front", "update")}
    L.castro_set_table_l2_window(1)
    return out


def run_batched_config(pkg, L, args, rank=0, world=1):
    """The batched configuration: a 256^3 Sedov domain on an uneven BoxArray (per-axis box sizes
    drawn from {16,24,32,48,64}) plus 32 independent instances of 32^3..96^3
    zones, advanced together; batched fused path and the one-launch step vs the per-box paths (per-routine
    sequence and drop-in).  With N
    ranks the instances are split over them by zone count (no data-path
    collective: instances are independent; strong scaling)."""
    import torch

    full = pkg.configs.batched()
    zones_all = [pkg.configs.zones(dict(full, instances=[i])) for i in full["instances"]]
    mine = pkg.replicas.partition_by_zones(zones_all, world)[rank] if world > 1 else list(range(len(zones_all)))
    cfg = dict(full, instances=[full["instances"][i] for i in mine])
    zones = sum(zones_all)
    out = {"workload": "batched: 256^3 uneven BoxArray + 32 instances 32^3..96^3, E 1e49-1e51, rho 0.1-10, 2 species",
           "zones": zones, "instances": len(full["instances"]),
           "boxes": sum(len(i["boxes"]) for i in full["instances"]),
           "sharding": (f"instances split over {world} ranks by zone count (largest first to the least-loaded "
                        "rank); no data-path collective" if world > 1 else "one GPU"),
           "scaling": "strong" if world > 1 else "single"}
    for mode, key, steps in ((pkg.castro.MODE_BATCHED, "batched", args.batched_steps),
                             (pkg.castro.MODE_PERSISTENT, "persistent", args.batched_steps),
                             (pkg.castro.MODE_PLAIN, "plain_per_box", 2),
                             (pkg.castro.MODE_PLAIN_BOX, "plain_box_drop_in", 2)):
        ms = 0.0
        launches = 0
        if cfg["instances"]:
            sim = pkg.make_sim(L, cfg, mode)
            sim.init_data()
            sim.step(2)
            sim.sync()
            st = torch.cuda.ExternalStream(sim.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            sim.step(steps)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            launches = sim.launches_per_step()
            sim.close()
        ms = pkg.replicas.max_over_ranks(ms, device="cuda")
        out[key] = {"value": zones * steps / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps,
                    "launches_per_step": launches}
    out["speedup_batched_over_plain"] = out["batched"]["value"] / out["plain_per_box"]["value"]
    out["speedup_batched_over_drop_in"] = out["batched"]["value"] / out["plain_box_drop_in"]["value"]
    out["persistent_over_batched"] = out["persistent"]["value"] / out["batched"]["value"]
    return out


WORKLOAD_TEXT = {
    "sedov128_pert": "128^3 zones in 64 boxes of 32^3, 2 species, outflow, rho=1*(1+1e-3 g), T=1e6 K, "
                     "E=1e50 erg in r=4 zones, CFL 0.5, 50 coarse steps",
    "sedov64": "one 64^3 box, 2 species, outflow, rho=1, T=1e6 K, E=1e50 erg in r=4 zones, 10 coarse steps",
    "large": "384^3 zones in an uneven BoxArray of 32^3..64^3 boxes, 2 species, outflow, rho=1*(1+1e-3 g), "
             "100 coarse steps",
    "adjoint64": "one 64^3 box, 2 species, outflow, rho=1*(1+1e-3 g), 20 coarse steps",
    "batched": "256^3 uneven BoxArray + 32 instances 32^3..96^3, 2 species, 20 coarse steps",
    "reference": "Source/Prob.F90 problem: 128^3 in 64^3 boxes, 13 species, periodic, 1e9 cm, 10 coarse steps",
}


def workload_text(args) -> str:
    t = f"{args.workload}: {WORKLOAD_TEXT.get(args.workload, '')}"
    return t + (f" (zone counts divided by {args.scale})" if args.scale > 1 else "")


def run_adjoint_config(pkg, args):
    """The gradient configuration: gradient of the shell kinetic energy (0.3 <= r/L <= 0.4) of a
    64^3 perturbed Sedov run over 20 steps with respect to the blast energy,
    the ambient density and the per-zone density perturbation, checkpoint every
    5 steps.  Reports forward and reverse device times (the forward is the
    reference launch sequence the reverse sweep recomputes; the fused batched
    forward of the same run is timed beside it) and central finite differences
    (relative step 1e-6) along 16 seeded directions."""
    import numpy as np
    import torch

    cfg = pkg.configs.adjoint64()
    inst = cfg["instances"][0]
    table = pkg.helm_table.ensure_table()
    L = pkg.castro.init(*cfg["network"], table)
    run = pkg.adjoint.SedovAdjoint(L, inst, cfg["steps"], cfg["checkpoint"], cfg["shell"])
    p = inst["problem"]
    E0, R0 = p["exp_energy"], p["dens_ambient"]
    pert0 = run.pert.clone()
    run.forward(E0, R0, pert0)                     # warm-up (allocations, first launches)
    run.backward()
    fwd_ms, bwd_ms = [], []
    for _ in range(max(1, args.adjoint_reps)):
        J0 = run.forward(E0, R0, pert0)
        dE, dR, dP = run.backward()
        f, b = run.time_ms()
        fwd_ms.append(f)
        bwd_ms.append(b)
    f_ms, b_ms = float(np.median(fwd_ms)), float(np.median(bwd_ms))
    # the same run through the fused batched forward (one CUDA graph per step)
    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    sim.sync()
    st = torch.cuda.ExternalStream(sim.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.step(cfg["steps"])
    e1.record(st)
    e1.synchronize()
    batched_ms = e0.elapsed_time(e1)
    sim.close()
    fd = None
    if args.adjoint_fd > 0:
        # 16 seeded directions: the blast energy alone, the ambient density alone, then random
        # combinations with the per-zone perturbation field.  The central difference is taken at
        # relative steps 1e-5, 1e-6 and 1e-7; a direction whose three differences agree to 1e-7 has
        # converged (no branch switch of a limiter or of the Riemann sampling inside the stencil).
        rng = np.random.default_rng(2019)
        n = run.n[0]
        zero = torch.zeros_like(pert0)
        dirs = [(1.0, 0.0, zero), (0.0, 1.0, zero)]
        for _ in range(max(0, args.adjoint_fd - 2)):
            a, b, c = rng.standard_normal(), rng.standard_normal(), rng.standard_normal((n, n, n))
            dirs.append((a, b, torch.from_numpy(np.ascontiguousarray(c.transpose(2, 1, 0))).cuda()))

        def fd_at(hh, a, b, ct):
            Jp = run.forward(E0 * (1 + hh * a), R0 * (1 + hh * b), pert0 + hh * ct)
            Jm = run.forward(E0 * (1 - hh * a), R0 * (1 - hh * b), pert0 - hh * ct)
            return (Jp - Jm) / (2 * hh)

        errs, spreads = [], []
        for a, b, ct in dirs[:args.adjoint_fd]:
            ad = dE * E0 * a + dR * R0 * b + float((dP * ct).sum())
            f5, f6, f7 = fd_at(1e-5, a, b, ct), fd_at(1e-6, a, b, ct), fd_at(1e-7, a, b, ct)
            sc = max(abs(f5), abs(f6), abs(f7))
            spreads.append(max(abs(f5 - f6), abs(f6 - f7), abs(f5 - f7)) / sc)
            errs.append(abs(ad - f6) / max(abs(ad), abs(f6)))
        conv = [e for e, sp in zip(errs, spreads) if sp <= 1e-7]
        fd = {"directions": len(errs), "relative_step": 1e-6, "max_rel_err": max(errs),
              "median_rel_err": float(np.median(errs)),
              "converged_directions": len(conv), "max_rel_err_converged": max(conv) if conv else None,
              "rel_errs": [float("%.3e" % e) for e in errs],
              "fd_step_spread": [float("%.3e" % e) for e in spreads],
              "note": "directions 0 and 1: blast energy alone, ambient density alone; fd_step_spread = largest "
                      "relative difference among the central differences at steps 1e-5, 1e-6, 1e-7; converged: "
                      "spread <= 1e-7"}
    out = {"workload": "adjoint64: 64^3 Sedov, perturbed density, 20 steps, checkpoint 5, shell 0.3-0.4",
           "J": J0, "dJ_dE": dE, "dJ_drho_ambient": dR, "dJ_dpert_norm": float(dP.norm()),
           "forward_ms": batched_ms, "backward_ms": b_ms, "adjoint_forward_ratio": b_ms / batched_ms,
           "ratio_note": "reverse sweep over the fused batched forward of the same 20 steps (one CUDA graph "
                         "per step); the reverse sweep recomputes its own forward in the per-box launch sequence",
           "per_box_forward_ms": f_ms, "backward_over_per_box_forward": b_ms / f_ms,
           "device_bytes": run.device_bytes(), "reps": len(fwd_ms), "fd_check": fd}
    run.close()
    return out


ORACLE_BUILDS = {
    "fast": "C oracle timing build (gcc -O3 -march=native, FMA contraction)",
    "parity": "C oracle parity build (gcc -O2 -ffp-contract=off)",
}


def time_oracle(pkg, workload, steps, warmup, variant):
    """Zone-updates/s of the oracle's level driver on all host cores: OpenMP
    over MFIter-style (1024,16,16) tiles as Source/Castro.cpp:26."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cfg = pkg.configs.WORKLOADS[workload]()
    A, Z = cfg["network"]
    table = pkg.helm_table.ensure_table()
    O.network_init(A, Z, variant)
    O.eos_init(table, variant)
    inst = cfg["instances"][0]
    lev, prob = O.level_from_instance(inst, pkg.configs.nvar(cfg), variant)
    cores = os.cpu_count() or 1
    lev.set_threads(cores)
    for _ in range(warmup):
        lev.coarse_step(-1.0)
    t0 = time.perf_counter()
    for _ in range(steps):
        lev.coarse_step(-1.0)
    t = time.perf_counter() - t0
    del lev
    return pkg.configs.zones(cfg) * steps / t, t, cores


def run_large_adjoint(pkg, slab_nz=32, first_step=50, nsteps=100, ckpt=5):
    """The large configuration's gradient: 384^3 Sedov with the seeded density
    perturbation, 100 steps of which the last 50 are differentiated (objective:
    the shell kinetic energy), checkpoint every 5 steps, each step reversed
    slab by slab (z-slabs of 32 zones) so that one slab's arrays are held.  Times
    the forward (all 100 steps) and the reverse sweep (the last 50)."""
    import torch

    cfg = pkg.configs.large()
    inst = cfg["instances"][0]
    table = pkg.helm_table.ensure_table()
    L = pkg.castro.init(*cfg["network"], table)
    torch.cuda.empty_cache()
    out = {"workload": "large: 384^3 Sedov, perturbed density, 100 steps, adjoint of the last 50, checkpoint 5, "
                       "shell 0.3-0.4", "slab_nz": slab_nz, "first_step": first_step}
    try:
        run = pkg.adjoint.SedovAdjoint(L, inst, nsteps, ckpt, (0.3, 0.4), slab_nz=slab_nz, first_step=first_step)
    except pkg.castro.CastroError as e:
        out["skipped"] = str(e)
        return out
    p = inst["problem"]
    J = run.forward(p["exp_energy"], p["dens_ambient"])
    run.backward()
    Vb = run.state_adjoint()
    f_ms, b_ms = run.time_ms()
    out.update({"J": J, "dJ_dV_norm": float(Vb.norm()), "forward_ms": f_ms, "backward_ms": b_ms,
                "backward_over_forward_of_the_window": b_ms / (f_ms * (nsteps - first_step) / nsteps),
                "device_bytes": run.device_bytes()})
    run.close()
    del Vb
    torch.cuda.empty_cache()
    return out


def cpu_baseline(pkg, args, steps=5):
    """Both oracle builds on the full workload: the timing build is the baseline's value."""
    out = {}
    for variant in ("fast", "parity"):
        v, t, cores = time_oracle(pkg, args.workload, steps, 1, variant)
        out[variant] = {"value": v, "seconds": t}
    return {"value": out["fast"]["value"], "unit": "zone-updates/s", "cores": cores, "kind": "port",
            "sample": f"{steps} coarse steps of the full {args.workload} level after one untimed step, "
                      f"{ORACLE_BUILDS['fast']} ({out['fast']['seconds']:.1f} s); OpenMP over (1024,16,16) tiles",
            "parity_build": {"value": out["parity"]["value"], "unit": "zone-updates/s",
                             "sample": f"the same {steps} steps, {ORACLE_BUILDS['parity']} "
                                       f"({out['parity']['seconds']:.1f} s)"}}


def run_reference(args, pkg):
    v, t, cores = time_oracle(pkg, args.workload, args.steps, args.warmup, "fast")
    zones = pkg.configs.zones(pkg.configs.WORKLOADS[args.workload]())
    table = pkg.helm_table.ensure_table()
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: Sedov blast, seeded Gaussian density perturbation, generated Helmholtz table",
        "config": {"workload": workload_text(args), "zones": zones,
                   "helm_table_sha256": pkg.helm_table.sha256(table)},
        "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full coarse steps after {args.warmup} warm-up steps; the reference "
                                   "(Fortran + AMReX) cannot be compiled in this image, so its C restatement runs: "
                                   f"{ORACLE_BUILDS['fast']}, OpenMP over MFIter-style (1024,16,16) tiles"},
        "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=45)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="sedov128_pert")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--batched-steps", type=int, default=18, help="timed steps of the batched configuration (0: skip)")
    ap.add_argument("--persistent-steps", type=int, default=20, help="timed steps of the one-launch persistent step (0: skip)")
    ap.add_argument("--column-tile-steps", type=int, default=10,
                    help="timed steps with riemann2 + riemann3 as one column-tile kernel (0: skip)")
    ap.add_argument("--large-steps", type=int, default=5, help="timed steps of the 384^3 configuration (0: skip)")
    ap.add_argument("--large-adjoint", type=int, default=1, help="the 384^3 configuration's 50-step adjoint (0: skip)")
    ap.add_argument("--adjoint-reps", type=int, default=3, help="timed forward+reverse runs of the adjoint configuration (0: skip)")
    ap.add_argument("--adjoint-fd", type=int, default=16, help="finite-difference directions of the gradient check (0: skip)")
    ap.add_argument("--fd-table-steps", type=int, default=10,
                    help="timed steps of the workload on the Fermi-Dirac table (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=int, default=1, help="divide the workload's zone counts (profiling runs only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    pkg = load_package()

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, pkg)), flush=True)
        return

    import torch

    if world > 1:
        import datetime

        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_b200(args, pkg, rank, world)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pkg, args)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
