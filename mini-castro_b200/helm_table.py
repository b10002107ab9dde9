"""Generator for ``helm_table.dat``, the Helmholtz free-energy table read by ``eos_init``.

The reference reads a 541 x 201 table (density index i fastest, temperature
index j slowest) of the electron free energy and its derivatives from
``helm_table.dat`` (Source/eos.F90:626-670).  The file itself is a large
third-party blob that the reference repository does not carry, so this module
writes a thermodynamically consistent replacement in exactly that layout:

* block 1, one record per (i, j): f, fd, ft, fdd, ftt, fdt, fddt, fdtt, fddtt
* block 2: dpdf, dpdfd, dpdft, dpdfdt
* block 3: ef, efd, eft, efdt
* block 4: xf, xfd, xft, xfdt

with the grid t(j) = 10**(3 + j*0.05) K and d(i) = 10**(-12 + i*0.05) g/cc
(Source/eos.F90:60-69).

Physics ("ideal-nd" table): a non-degenerate, non-relativistic ideal electron
gas per unit (ye * rho), i.e. the Sackur-Tetrode free energy

    f(d, T) = -N_A k T [ ln(n_Q(T) / (N_A d)) + 1 ],   n_Q = 2 (2 pi m_e k T / h^2)^(3/2)

so that p = d^2 df/dd = N_A k T d, s = -df/dT and c_v = 1.5 N_A k.  All
derivatives are analytic, so the biquintic interpolation in eos() reproduces
the node values exactly and the pressure family (linear in T) is reproduced
exactly everywhere.  A real Fermi-Dirac table can be dropped in unchanged.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np

IMAX, JMAX = 541, 201
TLO, THI, DLO, DHI = 3.0, 13.0, -12.0, 15.0

# constants of Source/eos.F90:129-133 plus the electron mass
H_PLANCK = 6.6260689633e-27
AVO = 6.0221417930e23
KERG = 1.380650424e-16
ME = 9.1093826e-28

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "helm_table.dat")


def grid():
    tstp = (THI - TLO) / float(JMAX - 1)
    dstp = (DHI - DLO) / float(IMAX - 1)
    t = 10.0 ** (TLO + np.arange(JMAX) * tstp)
    d = 10.0 ** (DLO + np.arange(IMAX) * dstp)
    return d, t


def ideal_nd_tables():
    """Return the 21 tables as (JMAX, IMAX) arrays in read order."""
    d1, t1 = grid()
    T, D = np.meshgrid(t1, d1, indexing="ij")  # shape (JMAX, IMAX): j slow, i fast
    nak = AVO * KERG
    nq = 2.0 * (2.0 * np.pi * ME * KERG * T / (H_PLANCK * H_PLANCK)) ** 1.5
    L = np.log(nq / (AVO * D))
    zero = np.zeros_like(T)
    f = -nak * T * (L + 1.0)
    fd = nak * T / D
    ft = -nak * (L + 2.5)
    fdd = -nak * T / (D * D)
    ftt = -1.5 * nak / T
    fdt = nak / D
    fddt = -nak / (D * D)
    fdtt = zero
    fddtt = zero
    dpdf = nak * T
    dpdfd = zero
    dpdft = nak + zero
    dpdfdt = zero
    ef = -L
    efd = 1.0 / D
    eft = -1.5 / T
    efdt = zero
    xf = AVO * D
    xfd = AVO + zero
    xft = zero
    xfdt = zero
    return [
        [f, fd, ft, fdd, ftt, fdt, fddt, fdtt, fddtt],
        [dpdf, dpdfd, dpdft, dpdfdt],
        [ef, efd, eft, efdt],
        [xf, xfd, xft, xfdt],
    ]


def write_table(path: str = DEFAULT_PATH) -> str:
    """Write the table to ``path`` (atomically) and return the path."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = f"{path}.tmp.{os.getpid()}"
    with open(tmp, "w") as fp:
        for block in ideal_nd_tables():
            cols = np.stack([b.reshape(-1) for b in block], axis=1)  # rows: j slow, i fast
            np.savetxt(fp, cols, fmt="%.17e")
    os.replace(tmp, path)
    return path


def ensure_table(path: str = DEFAULT_PATH) -> str:
    """Generate the table if it does not exist yet; return its path."""
    if not os.path.exists(path):
        write_table(path)
    return path


def sha256(path: str = DEFAULT_PATH) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as fp:
        for chunk in iter(lambda: fp.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


if __name__ == "__main__":
    import sys

    p = write_table(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_PATH)
    print(p, sha256(p))
