"""The oracle's counting build (oracle/op_count.cpp): the same arithmetic as the
parity build, bit for bit, with every floating-point operation counted.

Its per-zone counts of the reference algorithm (oracle/count_ops.py) are the
algorithmic FP64 work the FP64 roofline divides by.  Checked here: an exact
count of one routine by hand (divu: per node three 8-term differences, each
7 adds and 2 multiplies, and 2 adds to sum them; 3 divisions per call), and
one coarse step of a small level bitwise equal on both builds with counts
that repeat.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle as O


def test_divu_counted_by_hand():
    lo, hi = (0, 0, 0), (3, 2, 1)
    qlo, qhi = (-1, -1, -1), (4, 3, 2)
    rng = np.random.default_rng(3)
    q = np.asfortranarray(rng.standard_normal((6, 5, 4, 10)))
    div = np.zeros((4, 3, 2), order="F")
    dx = np.array([0.5, 0.25, 0.125])
    out = {}
    for variant in ("parity", "count"):
        d = np.zeros_like(div)
        O.op_counts_reset()
        O.lib(variant).oracle_divu(O.ivec(lo), O.ivec(hi), O.ptr(q), O.ivec(qlo), O.ivec(qhi), O.ptr(dx), O.ptr(d),
                                   O.ivec(lo), O.ivec(hi))
        out[variant] = d
    assert np.array_equal(out["parity"], out["count"])
    n = 4 * 3 * 2
    c = O.op_counts()
    assert c == dict(add=23 * n, mul=6 * n, div=3, sqrt=0, transcendental=0, compare=0, sign=0), c


def _step(pkg, table, variant):
    cfg = pkg.configs.sedov128_pert(scale=8, max_box=64)          # 16^3 in 8 boxes of 8^3
    A, Z = cfg["network"]
    O.network_init(A, Z, variant)
    O.eos_init(table, variant)
    L, _ = O.level_from_instance(cfg["instances"][0], 7 + len(A), variant)
    L.coarse_step(1e30)
    if variant == "count":
        O.op_counts_reset()
    L.coarse_step(1e30)
    counts = O.op_counts() if variant == "count" else None
    return O.assemble(L, cfg["instances"][0]), L.dt, counts


def test_counting_build_is_the_parity_arithmetic(pkg, table):
    U0, dt0, _ = _step(pkg, table, "parity")
    U1, dt1, c1 = _step(pkg, table, "count")
    U2, dt2, c2 = _step(pkg, table, "count")
    assert np.array_equal(U0, U1) and dt0 == dt1
    assert c1 == c2
    nz = 16 ** 3
    flops = (c1["add"] + c1["mul"] + c1["div"] + c1["sqrt"] + c1["transcendental"]) / nz
    print("ops per zone-update, 16^3 in 8 boxes:", {k: round(v / nz, 1) for k, v in c1.items()})
    # the per-box algorithm's ghost-zone work makes 8^3 boxes dearer (60k) than 32^3 boxes (27.8k)
    assert 4.0e4 < flops < 8.0e4
