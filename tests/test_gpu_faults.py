"""Failure detection, tested with faults made on the host (no GPU fault, trap or
hang): a truncated or missing Helmholtz table (eos_init's reader,
Source/eos.F90:637-670), a NaN-seeded state (EOS Newton solves that reach
their 100-iteration limit, Source/eos.F90:520-552, reported through
castro_last_error and the failure counter), and corrupt BoxArrays (rejected
by castro_sim_create before anything is allocated), and a grid-barrier wait of
the persistent step that cannot be satisfied (it gives up after its poll limit
and the host reads CASTRO_ERR_TIMEOUT).  Also: checkpoint / restart continues
a run bit for bit, and two runs from the same initial state are bitwise
identical (no races in the batched step).

NaN inputs are safe on the device by construction: table coordinates pass
through table_trunc, which maps NaN and infinities to a finite value before
they are clamped into the table, and every other index comes from zone
positions, never from state values.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_TABLE_IO, ERR_ARG, ERR_EOS, ERR_IO = 3, 5, 6, 7


def _lib(pkg, table, exact=False, net=None):
    A, Z = net or pkg.configs.NET2
    return pkg.castro.init(A, Z, table, exact=exact)


def test_truncated_and_missing_table(pkg, table, tmp_path):
    L = _lib(pkg, table)
    with open(table) as fp:
        head = [next(fp) for _ in range(50000)]          # the first block is 108,741 lines
    bad = tmp_path / "helm_table_truncated.dat"
    bad.write_text("".join(head))
    L.castro_clear_error()
    assert L.castro_eos_init_path(str(bad).encode()) == ERR_TABLE_IO
    assert L.castro_last_error() == ERR_TABLE_IO and b"truncated" in L.castro_error_string()
    L.castro_clear_error()
    with open(table) as fp:
        lines = fp.readlines()
    lines[10] = "not-a-number " + lines[10]              # a complete table with one bad token
    garbled = tmp_path / "helm_table_garbled.dat"
    garbled.write_text("".join(lines))
    del lines
    assert L.castro_eos_init_path(str(garbled).encode()) == ERR_TABLE_IO
    L.castro_clear_error()
    assert L.castro_eos_init_path(str(tmp_path / "absent.dat").encode()) == ERR_TABLE_IO
    assert b"cannot open" in L.castro_error_string()
    L.castro_clear_error()
    # the table loaded before stays in use: a sim still runs
    cfg = pkg.configs.sedov64(scale=8)
    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    sim.step(1)
    sim.sync()
    sim.close()


def test_nan_state_reported(pkg, table):
    L = _lib(pkg, table)
    K = pkg.castro
    cfg = pkg.configs.sedov64(scale=4)                   # one 16^3 box
    sim = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    sim.init_data()
    sim.sync()
    state = sim.download()
    assert sim.eos_failures() == 0
    state[5] = np.nan                                    # density of zone (5,0,0)
    sim.upload(state)
    L.castro_clear_error()
    sim.step(1)
    with pytest.raises(K.CastroError, match="castro error 6"):
        sim.sync()
    assert sim.eos_failures() > 0
    sim.sync()                                           # reported once, then cleared
    sim.close()


@pytest.mark.parametrize("case", ["overlap", "gap", "outside", "empty", "noncubic", "bc"])
def test_corrupt_boxarray_rejected(pkg, table, case):
    L = _lib(pkg, table)
    K = pkg.castro
    n = 16
    boxes = [((0, 0, 0), (7, 15, 15)), ((8, 0, 0), (15, 15, 15))]
    inst = pkg.configs.instance(n, boxes, bc=1)
    if case == "overlap":
        inst["boxes"] = [((0, 0, 0), (8, 15, 15)), ((8, 0, 0), (15, 15, 15))]
    elif case == "gap":
        inst["boxes"] = [((0, 0, 0), (6, 15, 15)), ((8, 0, 0), (15, 15, 15))]
    elif case == "outside":
        inst["boxes"] = [((0, 0, 0), (7, 15, 15)), ((8, 0, 0), (16, 15, 15))]
    elif case == "empty":
        inst["boxes"] = boxes + [((3, 3, 3), (2, 3, 3))]
    elif case == "noncubic":
        inst["probhi"] = (1.0, 1.0, 2.0)
    elif case == "bc":
        inst["bc"] = 7
    cfg = dict(name="corrupt", network=pkg.configs.NET2, steps=1, instances=[inst])
    L.castro_clear_error()
    with pytest.raises(K.CastroError, match="castro error 5"):
        pkg.make_sim(L, cfg, K.MODE_BATCHED)
    L.castro_clear_error()




@pytest.mark.parametrize("entry", ["castro_construct_hydro_source_box", "castro_construct_hydro_source_box_noalloc"])
@pytest.mark.parametrize("bad", ["sborder", "source", "flux"])
def test_box_entry_point_rejects_short_arrays(pkg, table, entry, bad):
    """An array that does not cover what the per-box call would touch (Sborder
    without 4 ghost zones, a source smaller than the box, a flux array smaller
    than the box's faces): CASTRO_ERR_ARG before anything is launched."""
    import ctypes as C

    import torch

    L = _lib(pkg, table)
    K = pkg.castro
    lo, hi = (0, 0, 0), (7, 7, 7)
    sblo, sbhi = [-4, -4, -4], [11, 11, 11]
    srlo, srhi = [0, 0, 0], [7, 7, 7]
    fo = [torch.zeros(9 * 9 * 8 * 8, dtype=torch.float64, device="cuda") for _ in range(3)]
    folo, fohi = [0] * 9, [8, 7, 7, 7, 8, 7, 7, 7, 8]
    if bad == "sborder":
        sbhi[2] = 10
    elif bad == "source":
        srhi[0] = 6
    else:
        fohi[4] = 7                       # the y-face array stops one face short
    sb = torch.ones(9 * 16 ** 3, dtype=torch.float64, device="cuda")
    src = torch.zeros(9 * 8 ** 3, dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * 3)(*[f.data_ptr() for f in fo])
    L.castro_clear_error()
    rc = getattr(L, entry)(K.ivec(lo), K.ivec(hi), C.c_void_p(sb.data_ptr()), K.ivec(sblo), K.ivec(sbhi),
                           C.c_void_p(src.data_ptr()), K.ivec(srlo), K.ivec(srhi), ptrs, (C.c_int * 9)(*folo),
                           (C.c_int * 9)(*fohi), K.ivec(lo), K.ivec(hi), K.dvec([1.0, 1.0, 1.0]), C.c_double(1e-6))
    assert rc == ERR_ARG, L.castro_error_string()
    L.castro_clear_error()
    torch.cuda.synchronize()
    assert float(src.abs().max()) == 0.0 and all(float(f.abs().max()) == 0.0 for f in fo)


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_checkpoint_restart_bitwise(pkg, table, tmp_path, exact):
    """3 steps, checkpoint, 2 more steps; a fresh sim restarted from the
    checkpoint takes the same 2 steps to the same bits.  With the exact build the
    restart also runs in the per-box mode, which reproduces the batched path bit
    for bit."""
    L = _lib(pkg, table, exact=exact)
    K = pkg.castro
    cfg = pkg.configs.batched(scale=8, ninst=2)          # uneven BoxArray + two instances
    a = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    a.init_data()
    a.step(3)
    ck = str(tmp_path / "chk")
    a.write_checkpoint(ck)
    a.step(2)
    ref = a.download()
    ref_t = [(a.time(i), a.dt(i), a.steps(i)) for i in range(len(cfg["instances"]))]
    a.close()
    modes = [K.MODE_BATCHED] + ([K.MODE_PLAIN] if exact else [])
    for mode in modes:
        b = pkg.make_sim(L, cfg, mode)
        b.read_checkpoint(ck)
        b.step(2)
        got = b.download()
        assert np.array_equal(got, ref), f"restart in mode {mode} differs"
        for i in range(len(cfg["instances"])):
            assert b.time(i) == ref_t[i][0] and b.steps(i) == ref_t[i][2]
            if mode == K.MODE_BATCHED:
                assert b.dt(i) == ref_t[i][1]
        b.close()
    # a mismatched sim and a damaged file are refused
    other = pkg.make_sim(L, pkg.configs.sedov64(scale=8), K.MODE_BATCHED)
    with pytest.raises(K.CastroError, match="castro error 5"):
        other.read_checkpoint(ck)
    other.close()
    st = os.path.join(ck, "State_00001")
    with open(st, "r+b") as fp:
        fp.truncate(os.path.getsize(st) - 8)
    c = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    with pytest.raises(K.CastroError, match="castro error 7"):
        c.read_checkpoint(ck)
    c.close()


@pytest.mark.parametrize("mode", [1, 2, 0, 3], ids=["batched", "plain_box", "plain", "persistent"])
def test_step_deterministic(pkg, table, mode):
    """Two runs from the same initial state agree bit for bit (production build):
    no race or order-dependent reduction in the step -- in the batched graph, in
    the per-box host sequences whose boxes run concurrently on four streams
    (per-stream scratch), and in the one-launch step's work queues."""
    L = _lib(pkg, table)
    cfg = pkg.configs.sedov128_pert(scale=4, max_box=8)   # 32^3 in 64 boxes
    out = []
    for _ in range(2):
        sim = pkg.make_sim(L, cfg, mode)
        sim.init_data()
        sim.step(5)
        out.append((sim.download(), sim.dt(0)))
        sim.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_persistent_wait_limit(pkg, table):
    """A grid barrier of the persistent step made to wait for one CTA more than
    exist (a condition set on the host) gives up after its poll limit: the
    launch ends, castro_sim_sync reports CASTRO_ERR_TIMEOUT, the sim refuses
    further steps, and the device stays usable -- a fresh sim then matches the
    ten-kernel graph bit for bit."""
    L = _lib(pkg, table)
    K = pkg.castro
    cfg = pkg.configs.sedov64(scale=4)
    sim = pkg.make_sim(L, cfg, K.MODE_PERSISTENT)
    sim.init_data()
    assert L.castro_sim_set_wait_limit(sim.h, 1 << 12, 2, 1) == 0
    L.castro_clear_error()
    sim.step(1)
    with pytest.raises(K.CastroError, match="castro error 8"):
        sim.sync()
    with pytest.raises(K.CastroError, match="castro error 8"):
        sim.step(1)
    sim.close()
    out = []
    for mode in (K.MODE_PERSISTENT, K.MODE_BATCHED):
        s2 = pkg.make_sim(L, cfg, mode)
        s2.init_data()
        s2.step(3)
        out.append(s2.download())
        s2.close()
    assert np.array_equal(out[0], out[1])
