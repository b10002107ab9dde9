"""Reader of the AMReX native plotfiles written by castro_sim_write_plotfile
(single level, one data file): returns the header fields and the level's data
assembled into one (nx, ny, nz, ncomp) array over the domain."""
from __future__ import annotations

import os
import re

import numpy as np


def _ints(txt: str):
    return [int(v) for v in re.findall(r"-?\d+", txt)]


def read_plotfile(path: str):
    with open(os.path.join(path, "Header")) as fp:
        lines = fp.read().splitlines()
    it = iter(lines)
    version = next(it)
    nc = int(next(it))
    names = [next(it) for _ in range(nc)]
    ndim = int(next(it))
    time = float(next(it))
    finest = int(next(it))
    plo = [float(v) for v in next(it).split()]
    phi = [float(v) for v in next(it).split()]
    next(it)                                    # refinement ratios (none on one level)
    dom = _ints(next(it))
    steps = int(next(it))
    dx = [float(v) for v in next(it).split()]
    hdr = dict(version=version, names=names, ndim=ndim, time=time, finest_level=finest, prob_lo=plo,
               prob_hi=phi, domain=(tuple(dom[0:3]), tuple(dom[3:6])), steps=steps, dx=dx)
    lo, hi = hdr["domain"]
    shape = tuple(h - l + 1 for l, h in zip(lo, hi))
    data = np.full(shape + (nc,), np.nan)
    with open(os.path.join(path, "Level_0", "Cell_H")) as fp:
        cell_h = fp.read().splitlines()
    offsets = [int(l.split()[2]) for l in cell_h if l.startswith("FabOnDisk:")]
    boxes = []
    with open(os.path.join(path, "Level_0", "Cell_D_00000"), "rb") as fp:
        raw = fp.read()
    for off in offsets:
        end = raw.index(b"\n", off)
        line = raw[off:end].decode()
        m = re.search(r"\)\)\)\((\(.*?\)) (\(.*?\)) \(.*?\)\) (\d+)$", line)
        blo, bhi, ncf = _ints(m.group(1)), _ints(m.group(2)), int(m.group(3))
        n = [h - l + 1 for l, h in zip(blo, bhi)]
        vals = np.frombuffer(raw, dtype="<f8", count=n[0] * n[1] * n[2] * ncf, offset=end + 1)
        fab = vals.reshape(ncf, n[2], n[1], n[0]).transpose(3, 2, 1, 0)
        sl = tuple(slice(l - d, h - d + 1) for l, h, d in zip(blo, bhi, lo))
        data[sl] = fab
        boxes.append((tuple(blo), tuple(bhi)))
    hdr["boxes"] = boxes
    return hdr, data
