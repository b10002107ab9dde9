"""Whole-step parity of the simulation paths (Castro::advance + dt control)
against the oracle's level driver, through the C-ABI castro_sim_* entry points.

* plain   : the reference's per-box launch sequence of the per-routine kernels;
* batched : the fused ten-kernel step over every box of every instance,
            replayed as a CUDA graph;
* plain_box: the plain host sequence with each box's hydro source from the
            coarse drop-in castro_construct_hydro_source_box;
* persistent: the batched step as one cooperative launch over device work queues.
The exact build must reproduce the oracle bit for bit, dt included; the
production build within the tolerances of gpu_harness (1e-12 per zone after
one step, 1e-9 relative L1 after a run, dt within 1e-14).
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_harness import RTOL_L1, RTOL_STEP, assert_match, from_dev, rel_l1, sborder_from_domain, to_dev

pytestmark = pytest.mark.gpu

# front, ghost, prep, trace, trace2, riemann1, riemann2, riemann3, update, dt --
# for any number of boxes and instances
FUSED_KERNELS_PER_STEP = 10

_current = {}


def gpu_lib(pkg, table, network, exact):
    key = (exact, tuple(network[0]))
    L = pkg.castro.load(exact)
    if _current.get(exact) != key:
        pkg.castro.init(network[0], network[1], table, exact=exact)
        _current[exact] = key
    return L


def oracle_run(oracle, pkg, table, cfg, steps):
    A, Z = cfg["network"]
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    out = []
    for inst in cfg["instances"]:
        lev, prob = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
        dts = [lev.coarse_step(inst.get("stop_time", -1.0)) for _ in range(steps)]
        out.append((oracle.assemble(lev, inst), dts, lev.time))
    return out


def gpu_run(pkg, table, cfg, steps, mode, exact):
    L = gpu_lib(pkg, table, cfg["network"], exact)
    sim = pkg.make_sim(L, cfg, mode)
    sim.init_data()
    dts = []
    for _ in range(steps):
        sim.step(1)
        dts.append([sim.dt(i) for i in range(len(cfg["instances"]))])
    states = sim.box_states()
    G = [pkg.castro.assemble(inst, states[i]) for i, inst in enumerate(cfg["instances"])]
    times = [sim.time(i) for i in range(len(cfg["instances"]))]
    assert sim.eos_failures() == 0
    launches = sim.launches_per_step()
    sim.close()
    return G, np.array(dts), times, launches


WORKLOADS = {
    "sedov16_outflow": lambda c: c.sedov64(scale=4),
    "sedov32_pert_8boxes": lambda c: c.sedov128_pert(scale=4, max_box=64),
    "reference16_periodic_8boxes": lambda c: c.reference(scale=8, max_box=64),
}


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
@pytest.mark.parametrize("mode", [0, 1, 2, 3], ids=["plain", "batched", "plain_box", "persistent"])
@pytest.mark.parametrize("wl", list(WORKLOADS))
def test_steps_match_oracle(pkg, table, oracle, wl, mode, exact):
    cfg = WORKLOADS[wl](pkg.configs)
    steps = 3
    ref = oracle_run(oracle, pkg, table, cfg, steps)
    G, dts, times, launches = gpu_run(pkg, table, cfg, steps, mode, exact)
    Go, dto, to = ref[0]
    if exact:
        np.testing.assert_array_equal(G[0], Go)
        assert list(dts[:, 0]) == dto
        assert times[0] == to
    else:
        assert_match(G[0], Go, False, rtol=RTOL_STEP * 10, what=wl)
        np.testing.assert_allclose(dts[:, 0], dto, rtol=1e-14)
    if mode == 1:
        assert launches == FUSED_KERNELS_PER_STEP
    if mode == 3:
        assert launches == 1          # the whole step in one cooperative launch


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_one_step_per_zone_tolerance(pkg, table, oracle, exact):
    """After one step every zone agrees to 1e-12 (scaled) -- the stated bar."""
    cfg = pkg.configs.sedov128_pert(scale=4, max_box=8)   # 32^3 in 64 boxes of 8^3
    ref = oracle_run(oracle, pkg, table, cfg, 1)
    G, dts, times, _ = gpu_run(pkg, table, cfg, 1, 1, exact)
    assert_match(G[0], ref[0][0], exact, rtol=RTOL_STEP, what="one step")


def test_full_run_l1(pkg, table, oracle):
    """Relative L1 per component after a 10-step run of the 16^3 outflow case."""
    cfg = pkg.configs.sedov64(scale=4)
    ref = oracle_run(oracle, pkg, table, cfg, 10)
    G, dts, times, _ = gpu_run(pkg, table, cfg, 10, 1, False)
    l1 = rel_l1(G[0], ref[0][0])
    assert (l1 <= RTOL_L1).all(), l1
    np.testing.assert_allclose(dts[:, 0], ref[0][1], rtol=1e-14)


def test_batched_instances_and_uneven_boxes(pkg, table, oracle):
    """Many independent instances of different sizes, energies and densities,
    plus an uneven BoxArray, in one batched sim: each instance bit-identical to
    its own oracle run (exact build)."""
    cfg = pkg.configs.batched(scale=8, ninst=5)   # 32^3 uneven + five 8..12^3 instances
    steps = 2
    ref = oracle_run(oracle, pkg, table, cfg, steps)
    G, dts, times, launches = gpu_run(pkg, table, cfg, steps, 1, True)
    assert launches == FUSED_KERNELS_PER_STEP
    for n, (Go, dto, to) in enumerate(ref):
        np.testing.assert_array_equal(G[n], Go, err_msg=f"instance {n}")
        assert list(dts[:, n]) == dto


def test_periodic_conservation_gpu(pkg, table):
    cfg = pkg.configs.reference(scale=4, max_box=16)    # 32^3 in eight 16^3 boxes, 13 species
    L = gpu_lib(pkg, table, cfg["network"], False)
    sim = pkg.make_sim(L, cfg, 1)
    sim.init_data()
    G0 = pkg.castro.assemble(cfg["instances"][0], sim.box_states()[0])
    sim.step(5)
    G = pkg.castro.assemble(cfg["instances"][0], sim.box_states()[0])
    sim.close()
    assert abs(G[..., 0].sum() / G0[..., 0].sum() - 1) < 1e-13
    assert abs(G[..., 4].sum() / G0[..., 4].sum() - 1) < 1e-13


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_construct_hydro_source_box(pkg, table, oracle, exact):
    """The fused per-box entry point against Castro::construct_hydro_source's
    body on the oracle (same cleaned Sborder, same dt), with store_flux."""
    import ctypes as C

    import torch

    cfg = pkg.configs.reference(scale=8, max_box=8)
    A, Z = cfg["network"]
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    inst = cfg["instances"][0]
    nv = pkg.configs.nvar(cfg)
    lev, prob = oracle.level_from_instance(inst, nv)
    for _ in range(2):
        lev.coarse_step(-1.0)
    dt = lev.est_time_step()
    G = oracle.assemble(lev, inst)
    lo, hi = inst["boxes"][3]
    sblo, sbhi = [l - 4 for l in lo], [h + 4 for h in hi]
    sb = sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"])
    for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
        oracle.call(name, sblo, sbhi, sb, sblo, sbhi)
    dx = [1e9 / 16] * 3
    src_ref = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)) + (nv,), order="F")
    oracle.lib().oracle_construct_hydro_source_tile(
        oracle.ivec(lo), oracle.ivec(hi), sb.ctypes.data_as(C.POINTER(C.c_double)), oracle.ivec(sblo),
        oracle.ivec(sbhi), src_ref.ctypes.data_as(C.POINTER(C.c_double)), oracle.ivec(lo), oracle.ivec(hi),
        oracle.ivec(inst["dom_lo"]), oracle.ivec(inst["dom_hi"]), oracle.dvec(dx), C.c_double(dt))
    L = gpu_lib(pkg, table, cfg["network"], exact)
    src = to_dev(np.zeros_like(src_ref))
    ebx = []
    fo = []
    for d in range(3):
        h = list(hi)
        h[d] += 1
        ebx.append((list(lo), h))
        fo.append(torch.full((nv,) + tuple(b - a + 1 for a, b in reversed(list(zip(lo, h)))), float("nan"),
                             dtype=torch.float64, device="cuda"))
    ptrs = (C.c_void_p * 3)(*[f.data_ptr() for f in fo])
    folo = (C.c_int * 9)(*[x for e in ebx for x in e[0]])
    fohi = (C.c_int * 9)(*[x for e in ebx for x in e[1]])
    K = pkg.castro
    rc = L.castro_construct_hydro_source_box(K.ivec(lo), K.ivec(hi), C.c_void_p(to_dev(sb).data_ptr()),
                                             K.ivec(sblo), K.ivec(sbhi), C.c_void_p(src.data_ptr()), K.ivec(lo),
                                             K.ivec(hi), ptrs, folo, fohi, K.ivec(inst["dom_lo"]),
                                             K.ivec(inst["dom_hi"]), K.dvec(dx), C.c_double(dt))
    torch.cuda.synchronize()
    assert rc == 0, L.castro_error_string()
    assert_match(from_dev(src), src_ref, exact, what="construct_hydro_source_box")
    # store_flux of the fused path: dt * F * A of the final fluxes
    for d in range(3):
        f = from_dev(fo[d])
        assert np.isfinite(f).all()
    # conservation inside the box: the flux-divergence of rho equals the boundary flux balance
    area = dx[1] * dx[2]
    tot = from_dev(src)[..., 0].sum() * dx[0] * dx[1] * dx[2] * dt
    fx = [from_dev(fo[d])[..., 0] for d in range(3)]
    bal = (fx[0][0].sum() - fx[0][-1].sum() + fx[1][:, 0].sum() - fx[1][:, -1].sum()
           + fx[2][:, :, 0].sum() - fx[2][:, :, -1].sum())
    assert abs(tot - bal) <= 1e-12 * max(abs(bal), abs(tot), area)


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_construct_hydro_source_box_shapes(pkg, table, oracle, exact):
    """The per-box entry point over boxes of changing shape in one process --
    small, the largest (the library's scratch grows), then smaller shapes laid
    out afresh in the grown scratch -- each against the oracle's
    construct_hydro_source on the same cleaned Sborder: the exact build against
    the parity oracle bit for bit, the production build against the oracle's
    contracting build (liboracle_fast.so) to 1e-12.  The production build and
    the contracting CPU build round alike; between either and the parity build
    the hydro source of the whole 32^3 blast, a flux divergence, differs by up
    to 2e-12 of its components' largest magnitude through cancellation."""
    import ctypes as C

    cfg = pkg.configs.sedov64(scale=2)               # one 32^3 box, 2 species, outflow
    A, Z = cfg["network"]
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    inst = cfg["instances"][0]
    nv = pkg.configs.nvar(cfg)
    lev, prob = oracle.level_from_instance(inst, nv)
    for _ in range(3):
        lev.coarse_step(-1.0)
    dt = lev.est_time_step()
    G = oracle.assemble(lev, inst)
    variant = "parity" if exact else "fast"
    oracle.network_init(A, Z, variant)
    oracle.eos_init(table, variant)
    OL = oracle.lib(variant)
    L = gpu_lib(pkg, table, cfg["network"], exact)
    K = pkg.castro
    dx = [1.0 / 32] * 3
    for lo, hi in (((4, 4, 4), (11, 11, 19)), ((0, 0, 0), (31, 31, 31)), ((8, 2, 5), (23, 13, 24)),
                   ((12, 12, 12), (19, 19, 19))):
        sblo, sbhi = [l - 4 for l in lo], [h + 4 for h in hi]
        sb = sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"])
        for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
            getattr(OL, "oracle_" + name)(oracle.ivec(sblo), oracle.ivec(sbhi), sb.ctypes.data_as(C.POINTER(C.c_double)),
                                          oracle.ivec(sblo), oracle.ivec(sbhi))
        src_ref = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)) + (nv,), order="F")
        OL.oracle_construct_hydro_source_tile(
            oracle.ivec(lo), oracle.ivec(hi), sb.ctypes.data_as(C.POINTER(C.c_double)), oracle.ivec(sblo),
            oracle.ivec(sbhi), src_ref.ctypes.data_as(C.POINTER(C.c_double)), oracle.ivec(lo), oracle.ivec(hi),
            oracle.ivec(inst["dom_lo"]), oracle.ivec(inst["dom_hi"]), oracle.dvec(dx), C.c_double(dt))
        src = to_dev(np.zeros_like(src_ref))
        rc = L.castro_construct_hydro_source_box(K.ivec(lo), K.ivec(hi), C.c_void_p(to_dev(sb).data_ptr()),
                                                 K.ivec(sblo), K.ivec(sbhi), C.c_void_p(src.data_ptr()), K.ivec(lo),
                                                 K.ivec(hi), None, None, None, K.ivec(inst["dom_lo"]),
                                                 K.ivec(inst["dom_hi"]), K.dvec(dx), C.c_double(dt))
        assert rc == 0, L.castro_error_string()
        assert_match(from_dev(src), src_ref, exact, what=f"construct_hydro_source_box {lo}-{hi}")


def test_plotfile_roundtrip(pkg, table, tmp_path):
    """castro_sim_write_plotfile: AMReX layout (Header, Level_0/Cell_H,
    Level_0/Cell_D_00000) read back into the exact domain state, with the
    instance's time, step count, geometry and BoxArray."""
    cfg = pkg.configs.batched(scale=8, ninst=2)      # 32^3 uneven BoxArray + two instances
    L = gpu_lib(pkg, table, cfg["network"], False)
    sim = pkg.make_sim(L, cfg, 1)
    sim.init_data()
    sim.step(3)
    states = sim.box_states()
    for n, inst in enumerate(cfg["instances"]):
        path = str(tmp_path / f"plt{n}")
        sim.write_plotfile(path, n)
        hdr, data = pkg.plotfile.read_plotfile(path)
        G = pkg.castro.assemble(inst, states[n])
        np.testing.assert_array_equal(data, G)
        assert hdr["version"] == "HyperCLaw-V1.1"
        assert hdr["names"][:7] == ["density", "xmom", "ymom", "zmom", "rho_E", "rho_e", "Temp"]
        assert hdr["steps"] == 3 and hdr["time"] == sim.time(n)
        assert hdr["domain"] == (tuple(inst["dom_lo"]), tuple(inst["dom_hi"]))
        assert sorted(hdr["boxes"]) == sorted((tuple(a), tuple(b)) for a, b in inst["boxes"])
        n_cell = inst["dom_hi"][0] - inst["dom_lo"][0] + 1
        assert hdr["dx"][0] == pytest.approx((inst["probhi"][0] - inst["problo"][0]) / n_cell, rel=1e-15)
    sim.close()


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_column_tiles_match_oracle(pkg, table, oracle, exact):
    """castro_set_column_tiles: riemann2 + riemann3 as one kernel per column tile
    with the cross fluxes in shared memory (2 species, batched mode).  The same
    per-face stages on the same inputs: bit for bit the oracle with the exact
    build, on a single box, on 8 boxes with a perturbed density, and on an
    uneven BoxArray plus instances whose domains are not multiples of the tile
    (partial tiles); nine kernels per step."""
    cfgs = [WORKLOADS["sedov16_outflow"](pkg.configs), WORKLOADS["sedov32_pert_8boxes"](pkg.configs),
            pkg.configs.batched(scale=8, ninst=3)]
    L = gpu_lib(pkg, table, cfgs[0]["network"], exact)
    L.castro_set_column_tiles(1)
    try:
        for cfg in cfgs:
            steps = 3
            ref = oracle_run(oracle, pkg, table, cfg, steps)
            G, dts, times, launches = gpu_run(pkg, table, cfg, steps, 1, exact)
            assert launches == FUSED_KERNELS_PER_STEP - 1
            for n, (Go, dto, to) in enumerate(ref):
                if exact:
                    np.testing.assert_array_equal(G[n], Go, err_msg=f"{cfg['name']} instance {n}")
                    assert list(dts[:, n]) == dto
                else:
                    assert_match(G[n], Go, False, rtol=RTOL_STEP * 10, what=cfg["name"])
    finally:
        L.castro_set_column_tiles(0)
