"""castro_construct_hydro_source_box_noalloc against castro_construct_hydro_source_box.

The no-allocation entry point serves callers that cannot allocate device
memory while they advance a box (hosts that own all device memory through a
pool reserved at start-up, hosts that may not call cudaMalloc inside a time
step because it synchronizes the device).  It keeps its scratch in one static
device array of the library, so this test calls it twice in a row on
different boxes and time steps -- the second call must not see anything the
first one left behind -- and checks both against the allocating entry point
through the C-ABI, within the tolerance of the other kernel tests.  It also
checks that a box larger than the array is refused before any launch.

Self-contained: it builds its own input state with the library, so it passes
in a fresh process as well as after the rest of the suite.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_harness import RTOL_KERNEL, assert_match, from_dev, sborder_from_domain, to_dev

pytestmark = pytest.mark.gpu


def _state(pkg, table):
    """A 16^3 reference-problem state (13 species, periodic) after two steps."""
    cfg = pkg.configs.reference(scale=8, max_box=8)
    A, Z = cfg["network"]
    L = pkg.castro.init(A, Z, table)
    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    sim.step(2)
    inst = cfg["instances"][0]
    G = pkg.castro.assemble(inst, sim.box_states()[0])
    dt = sim.est_time_step()
    sim.close()
    return L, cfg, inst, G, dt


def _call(L, K, fn, lo, hi, sb, sblo, sbhi, nv, dx, dt):
    import torch

    src = torch.zeros((nv,) + tuple(h - l + 1 for l, h in reversed(list(zip(lo, hi)))), dtype=torch.float64,
                      device="cuda")
    fo, los, his = [], [], []
    for d in range(3):
        h = list(hi)
        h[d] += 1
        los += list(lo)
        his += h
        fo.append(torch.full((nv,) + tuple(b - a + 1 for a, b in reversed(list(zip(lo, h)))), float("nan"),
                             dtype=torch.float64, device="cuda"))
    ptrs = (C.c_void_p * 3)(*[f.data_ptr() for f in fo])
    rc = getattr(L, fn)(K.ivec(lo), K.ivec(hi), C.c_void_p(sb.data_ptr()), K.ivec(sblo), K.ivec(sbhi),
                        C.c_void_p(src.data_ptr()), K.ivec(lo), K.ivec(hi), ptrs, (C.c_int * 9)(*los),
                        (C.c_int * 9)(*his), K.ivec((0, 0, 0)), K.ivec((15, 15, 15)), K.dvec(dx), C.c_double(dt))
    torch.cuda.synchronize()
    return rc, from_dev(src), [from_dev(f) for f in fo]


def test_noalloc_matches_allocating_entry_point(pkg, table):
    L, cfg, inst, G, dt = _state(pkg, table)
    K = pkg.castro
    nv = pkg.configs.nvar(cfg)
    dx = [1e9 / 16] * 3
    # two calls in a row on different boxes and time steps
    for box, dtc in ((3, dt), (6, 0.5 * dt)):
        lo, hi = inst["boxes"][box]
        sblo, sbhi = [l - 4 for l in lo], [h + 4 for h in hi]
        sbn = sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"])
        sb = to_dev(sbn)
        for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
            K.call(L, name, sblo, sbhi, sb, sblo, sbhi)
        rc0, src0, fo0 = _call(L, K, "castro_construct_hydro_source_box", lo, hi, sb, sblo, sbhi, nv, dx, dtc)
        rc1, src1, fo1 = _call(L, K, "castro_construct_hydro_source_box_noalloc", lo, hi, sb, sblo, sbhi, nv, dx, dtc)
        assert rc0 == 0 and rc1 == 0, L.castro_error_string()
        assert np.isfinite(src1).all()
        assert_match(src1, src0, False, rtol=RTOL_KERNEL, what=f"noalloc source, box {box}")
        for d in range(3):
            assert_match(fo1[d], fo0[d], False, rtol=RTOL_KERNEL, what=f"noalloc store_flux d={d}, box {box}")


def test_noalloc_rejects_oversized_box(pkg, table):
    import torch

    A, Z = pkg.configs.NET13
    L = pkg.castro.init(A, Z, table)
    K = pkg.castro
    lo, hi = (0, 0, 0), (23, 23, 23)     # 24^3 zones with 13 species: beyond the static array
    sblo, sbhi = (-4, -4, -4), (27, 27, 27)
    sb = torch.zeros(20 * 32 ** 3, dtype=torch.float64, device="cuda")
    src = torch.zeros(20 * 24 ** 3, dtype=torch.float64, device="cuda")
    L.castro_clear_error()
    rc = L.castro_construct_hydro_source_box_noalloc(K.ivec(lo), K.ivec(hi), C.c_void_p(sb.data_ptr()),
                                                     K.ivec(sblo), K.ivec(sbhi), C.c_void_p(src.data_ptr()),
                                                     K.ivec(lo), K.ivec(hi), None, None, None, K.ivec(lo),
                                                     K.ivec(hi), K.dvec([1.0, 1.0, 1.0]), C.c_double(1e-3))
    assert rc == 5                               # CASTRO_ERR_ARG
    assert b"static array" in L.castro_error_string()
    L.castro_clear_error()
    torch.cuda.synchronize()
    assert float(src.abs().max()) == 0.0         # nothing was launched


def test_noalloc_shape_changes_and_capacity(pkg, table):
    """Calls in a row whose box shapes differ (8x8x16, then 21^3, then 8^3), so the
    layout carved out of the static array moves between calls, each against the
    allocating entry point; 21^3 with 2 species is the largest cube the array
    holds and 22^3 is refused."""
    cfg = pkg.configs.sedov64(scale=2)               # one 32^3 box, 2 species, outflow
    A, Z = cfg["network"]
    L = pkg.castro.init(A, Z, table)
    K = pkg.castro
    sim = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    sim.init_data()
    sim.step(3)
    inst = cfg["instances"][0]
    G = K.assemble(inst, sim.box_states()[0])
    dt = sim.est_time_step()
    sim.close()
    nv = pkg.configs.nvar(cfg)
    dx = [1.0 / 32] * 3
    for lo, hi, dtc in (((4, 4, 4), (11, 11, 19), dt), ((5, 5, 5), (25, 25, 25), 0.7 * dt), ((12, 12, 12), (19, 19, 19), dt)):
        sblo, sbhi = [l - 4 for l in lo], [h + 4 for h in hi]
        sb = to_dev(sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"]))
        for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
            K.call(L, name, sblo, sbhi, sb, sblo, sbhi)
        rc0, src0, fo0 = _call(L, K, "castro_construct_hydro_source_box", lo, hi, sb, sblo, sbhi, nv, dx, dtc)
        rc1, src1, fo1 = _call(L, K, "castro_construct_hydro_source_box_noalloc", lo, hi, sb, sblo, sbhi, nv, dx, dtc)
        assert rc0 == 0 and rc1 == 0, L.castro_error_string()
        assert np.isfinite(src1).all()
        assert_match(src1, src0, False, rtol=RTOL_KERNEL, what=f"noalloc source, box {lo}-{hi}")
        for d in range(3):
            assert_match(fo1[d], fo0[d], False, rtol=RTOL_KERNEL, what=f"noalloc store_flux d={d}, box {lo}-{hi}")
    lo, hi = (4, 4, 4), (25, 25, 25)                 # 22^3 with 2 species: one zone per side too many
    sblo, sbhi = [l - 4 for l in lo], [h + 4 for h in hi]
    sb = to_dev(sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"]))
    L.castro_clear_error()
    rc, src, _ = _call(L, K, "castro_construct_hydro_source_box_noalloc", lo, hi, sb, sblo, sbhi, nv, dx, dt)
    assert rc == 5 and b"static array" in L.castro_error_string()
    L.castro_clear_error()
    assert float(np.abs(src).max()) == 0.0
