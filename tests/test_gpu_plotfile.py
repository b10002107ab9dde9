"""castro_sim_write_plotfile against AMReX's native plotfile grammar, checked
line by line by a parser of its own (not mini-castro_b200/plotfile.py; the
image has no AMReX or yt reader to hand it to).

The layout AMReX's plotfile writer and VisMF produce for one level, one data
file:

Header                  "HyperCLaw-V1.1", ncomp, ncomp names, spacedim 3, time,
                        finest level 0, prob_lo, prob_hi, the (empty) line of
                        refinement ratios, the domain box "((lo) (hi) (0,0,0))",
                        the level's steps, its cell size, coordinate system 0,
                        boundary width 0, then per level "lev nboxes time",
                        steps, each box's physical [lo, hi] per direction, and
                        the MultiFab's path "Level_0/Cell"
Level_0/Cell_H          VisMF header version 1, "how" 0, ncomp, ngrow 0, the
                        BoxArray "(n 0" ... ")", n, one "FabOnDisk: file offset"
                        per box, then the per-box minima and maxima of every
                        component ("n,ncomp" and one comma-terminated row per box)
Level_0/Cell_D_00000    per box a FAB header line naming the IEEE double format
                        (64 11 52 0 1 12 0 1023) and the little-endian byte order
                        (8 7 6 5 4 3 2 1), the box and ncomp, then the values in
                        Fortran order, component slowest
"""
from __future__ import annotations

import os
import re
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOX = r"\(\((-?\d+),(-?\d+),(-?\d+)\) \((-?\d+),(-?\d+),(-?\d+)\) \(0,0,0\)\)"
FAB = re.compile(rb"FAB \(\(8, \(64 11 52 0 1 12 0 1023\)\),\(8, \(8 7 6 5 4 3 2 1\)\)\)" + BOX.encode()
                 + rb" (\d+)\n")


def _floats(line, n):
    v = [float(x) for x in line.split()]
    assert len(v) == n, line
    return v


def check_plotfile(path, inst, state_boxes, time, steps, nvar):
    """Parse path strictly; return the domain data it holds."""
    lines = open(os.path.join(path, "Header")).read().split("\n")
    assert lines[-1] == "" and lines[-2] == "Level_0/Cell"
    it = iter(lines)
    assert next(it) == "HyperCLaw-V1.1"
    assert int(next(it)) == nvar
    names = [next(it) for _ in range(nvar)]
    assert names[:7] == ["density", "xmom", "ymom", "zmom", "rho_E", "rho_e", "Temp"]
    assert all(re.fullmatch(r"[A-Za-z_][A-Za-z0-9_]*", n) for n in names) and len(set(names)) == nvar
    assert next(it) == "3"
    assert float(next(it)) == time
    assert next(it) == "0"
    plo, phi = _floats(next(it), 3), _floats(next(it), 3)
    assert plo == list(inst["problo"]) and phi == list(inst["probhi"])
    assert next(it) == ""                                   # no refinement ratios on one level
    m = re.fullmatch(BOX, next(it))
    lo, hi = [int(x) for x in m.groups()[:3]], [int(x) for x in m.groups()[3:]]
    assert (tuple(lo), tuple(hi)) == (tuple(inst["dom_lo"]), tuple(inst["dom_hi"]))
    assert int(next(it)) == steps
    dx = _floats(next(it), 3)
    for d in range(3):
        assert dx[d] == pytest.approx((phi[d] - plo[d]) / (hi[d] - lo[d] + 1), rel=1e-15)
    assert next(it) == "0" and next(it) == "0"              # Cartesian, no boundary data
    lev, nbox, t = next(it).split()
    assert lev == "0" and int(nbox) == len(inst["boxes"]) and float(t) == time
    assert int(next(it)) == steps
    hdr_boxes = []
    for _ in range(int(nbox)):
        ext = [_floats(next(it), 2) for _ in range(3)]
        blo = [round((ext[d][0] - plo[d]) / dx[d]) for d in range(3)]
        bhi = [round((ext[d][1] - plo[d]) / dx[d]) - 1 for d in range(3)]
        for d in range(3):
            assert ext[d][0] == pytest.approx(plo[d] + blo[d] * dx[d], rel=1e-14, abs=1e-300)
        hdr_boxes.append((tuple(blo), tuple(bhi)))
    assert next(it) == "Level_0/Cell"

    ch = open(os.path.join(path, "Level_0", "Cell_H")).read().split("\n")
    it = iter(ch)
    assert next(it) == "1" and next(it) == "0"
    assert int(next(it)) == nvar and next(it) == "0"
    assert next(it) == f"({nbox} 0"
    ba = []
    for _ in range(int(nbox)):
        m = re.fullmatch(BOX, next(it))
        g = [int(x) for x in m.groups()]
        ba.append((tuple(g[:3]), tuple(g[3:])))
    assert next(it) == ")" and int(next(it)) == int(nbox)
    assert ba == hdr_boxes
    offs = []
    for _ in range(int(nbox)):
        tag, fname, off = next(it).split()
        assert tag == "FabOnDisk:" and fname == "Cell_D_00000"
        offs.append(int(off))
    mins, maxs = [], []
    for dest in (mins, maxs):
        assert next(it) == "" and next(it) == f"{nbox},{nvar}"
        for _ in range(int(nbox)):
            row = next(it)
            assert row.endswith(",")
            dest.append([float(x) for x in row[:-1].split(",")])
            assert len(dest[-1]) == nvar

    raw = open(os.path.join(path, "Level_0", "Cell_D_00000"), "rb").read()
    shape = tuple(h - l + 1 for l, h in zip(lo, hi))
    data = np.full(shape + (nvar,), np.nan)
    pos = 0
    for b, off in enumerate(offs):
        assert off == pos                                  # FABs back to back, in BoxArray order
        m = FAB.match(raw, off)
        g = [int(x) for x in m.groups()]
        assert (tuple(g[:3]), tuple(g[3:6])) == ba[b] and g[6] == nvar
        n = [g[3 + d] - g[d] + 1 for d in range(3)]
        cnt = n[0] * n[1] * n[2] * nvar
        vals = struct.unpack_from("<%dd" % cnt, raw, m.end())
        fab = np.array(vals).reshape(nvar, n[2], n[1], n[0]).transpose(3, 2, 1, 0)
        np.testing.assert_array_equal(fab, state_boxes[b])
        assert [fab[..., c].min() for c in range(nvar)] == mins[b]
        assert [fab[..., c].max() for c in range(nvar)] == maxs[b]
        data[tuple(slice(g[d] - lo[d], g[3 + d] - lo[d] + 1) for d in range(3))] = fab
        pos = m.end() + 8 * cnt
    assert pos == len(raw)
    assert not np.isnan(data).any()                        # the boxes tile the domain
    return data


def test_plotfile_amrex_grammar(pkg, table, tmp_path):
    cfg = pkg.configs.batched(scale=8, ninst=2)            # 32^3 uneven BoxArray + two instances
    nvar = pkg.configs.nvar(cfg)
    L = pkg.castro.init(*cfg["network"], table, exact=False)
    sim = pkg.make_sim(L, cfg, 1)
    sim.init_data()
    sim.step(2)
    states = sim.box_states()
    for n, inst in enumerate(cfg["instances"]):
        path = str(tmp_path / f"plt{n:05d}")
        sim.write_plotfile(path, n)
        data = check_plotfile(path, inst, states[n], sim.time(n), 2, nvar)
        np.testing.assert_array_equal(data, pkg.castro.assemble(inst, states[n]))
    sim.close()
