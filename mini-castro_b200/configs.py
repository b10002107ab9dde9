"""Sedov workloads: BoxArrays, species networks, problem constants, perturbations.

Each workload is a list of *instances*; an instance is one single-level Sedov
problem (domain, BoxArray, boundary condition, problem constants).  The same
description drives the GPU library and the CPU oracle.

Workloads (sizes as named by the benchmark configurations):

* ``sedov64``       -- one 64^3 box, unit cube, outflow, two species, rho=1, T=1e6 K,
                       E=1e50 erg in a sphere of 4 zones, 10 steps (reference CPU case).
* ``sedov128_pert`` -- 128^3 in 64 boxes of 32^3, density times (1+1e-3 g) with g a
                       seeded unit-variance Gaussian field smoothed over 4 zones, 50 steps.
* ``batched``       -- 256^3 cut into an uneven BoxArray (per-axis sizes drawn from
                       {16,24,32,48,64}) plus 32 independent instances of 32^3..96^3
                       zones with log-uniform energies and ambient densities, 20 steps.
* ``adjoint64``     -- one 64^3 box with the seeded perturbation, 20 steps: the
                       gradient case (objective: kinetic energy in the shell
                       0.3 <= r/L <= 0.4; checkpoint every 5 steps).
* ``large``         -- 384^3 in boxes of 32^3..64^3 with the perturbation, 100 steps.
* ``reference``     -- the Source/Prob.F90 problem (13 species, periodic, 1e9 cm
                       domain), the physically in-table case.

Every workload takes a ``scale`` divisor so tests can run the same shapes small.
"""
from __future__ import annotations

import math

import numpy as np

NET2 = ([4.0, 16.0], [2.0, 8.0])
NET13 = ([4., 12., 16., 20., 24., 28., 32., 36., 40., 44., 48., 52., 56.],
         [2., 6., 8., 10., 12., 14., 16., 18., 20., 22., 24., 26., 28.])


def chop(n: int, max_size: int) -> list[int]:
    """Split n zones into ceil(n/max_size) pieces of near-equal size."""
    k = max(1, -(-n // max_size))
    base, rem = divmod(n, k)
    return [base + (1 if i < rem else 0) for i in range(k)]


def boxes_from_sizes(sx, sy, sz, lo=(0, 0, 0)):
    boxes = []
    z0 = lo[2]
    for nz in sz:
        y0 = lo[1]
        for ny in sy:
            x0 = lo[0]
            for nx in sx:
                boxes.append(((x0, y0, z0), (x0 + nx - 1, y0 + ny - 1, z0 + nz - 1)))
                x0 += nx
            y0 += ny
        z0 += nz
    return boxes


def uniform_boxes(n: int, max_box: int):
    s = chop(n, max_box)
    return boxes_from_sizes(s, s, s)


def uneven_sizes(n: int, choices, rng) -> list[int]:
    """Seeded per-axis segment sizes from `choices` summing exactly to n."""
    choices = sorted(choices)
    for _ in range(1000):
        out, tot = [], 0
        while tot < n:
            rem = n - tot
            fit = [c for c in choices if c <= rem]
            if not fit:
                break
            if rem in choices and rng.random() < 0.5:
                c = rem
            else:
                c = int(rng.choice(fit))
            out.append(c)
            tot += c
        if tot == n:
            return out
    raise ValueError(f"cannot tile {n} with {choices}")


def gaussian_field(shape, sigma: float, seed: int) -> np.ndarray:
    """Seeded standard-normal field, periodic Gaussian smoothing of width sigma
    zones, renormalised to zero mean and unit variance (Fortran order)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kx, ky, kz = np.meshgrid(*k, indexing="ij")
    filt = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx * kx + ky * ky + kz * kz))
    f = np.real(np.fft.ifftn(np.fft.fftn(g) * filt))
    f = (f - f.mean()) / f.std()
    return np.asfortranarray(f)


def problem(**kw) -> dict:
    p = dict(ambient_from_T=1, dens_ambient=1.0, p_ambient=1e21, T_ambient=1e6, exp_energy=1e50,
             r_init=None, nsub=10, X=[0.5, 0.5], T_init=1e9, pert=None, pert_amp=0.0)
    p.update(kw)
    return p


def instance(n, boxes, *, bc=1, length=1.0, prob=None, lo=(0, 0, 0)):
    dx = length / n
    prob = dict(prob or problem())
    if prob["r_init"] is None:
        prob["r_init"] = 4.0 * dx
    return dict(dom_lo=tuple(lo), dom_hi=tuple(l + n - 1 for l in lo), problo=(0.0, 0.0, 0.0),
                probhi=(length,) * 3, bc=bc, boxes=boxes, problem=prob, n=n)


def sedov64(scale: int = 1, steps: int = 10):
    n = 64 // scale
    return dict(name="sedov64", network=NET2, steps=steps,
                instances=[instance(n, uniform_boxes(n, n), bc=1)])


def sedov128_pert(scale: int = 1, steps: int = 50, seed: int = 20191219, max_box: int = 32):
    n = 128 // scale
    mb = max(4, max_box // scale)
    pert = gaussian_field((n, n, n), 4.0, seed)
    prob = problem(pert=pert, pert_amp=1e-3)
    return dict(name="sedov128_pert", network=NET2, steps=steps,
                instances=[instance(n, uniform_boxes(n, mb), bc=1, prob=prob)])


def batched(scale: int = 1, steps: int = 20, seed: int = 7, ninst: int = 32):
    rng = np.random.default_rng(seed)
    n = 256 // scale
    choices = [c // scale for c in (16, 24, 32, 48, 64) if c // scale >= 4]
    sizes = [uneven_sizes(n, choices, rng) for _ in range(3)]
    insts = [instance(n, boxes_from_sizes(*sizes), bc=1)]
    for _ in range(ninst):
        m = int(rng.integers(32, 97)) // scale
        m = max(m, 8)
        E = 10.0 ** rng.uniform(49.0, 51.0)
        rho = 10.0 ** rng.uniform(-1.0, 1.0)
        insts.append(instance(m, uniform_boxes(m, 64 // scale if scale > 1 else 64), bc=1,
                              prob=problem(exp_energy=E, dens_ambient=rho)))
    return dict(name="batched", network=NET2, steps=steps, instances=insts)


def adjoint64(scale: int = 1, steps: int = 20, seed: int = 64):
    n = 64 // scale
    pert = gaussian_field((n, n, n), 4.0, seed)
    prob = problem(pert=pert, pert_amp=1e-3)
    return dict(name="adjoint64", network=NET2, steps=steps, checkpoint=5, shell=(0.3, 0.4),
                instances=[instance(n, uniform_boxes(n, n), bc=1, prob=prob)])


def large(scale: int = 1, steps: int = 100, seed: int = 384):
    rng = np.random.default_rng(seed)
    n = 384 // scale
    choices = [c // scale for c in (32, 48, 64) if c // scale >= 4]
    sizes = [uneven_sizes(n, choices, rng) for _ in range(3)]
    pert = gaussian_field((n, n, n), 4.0, seed)
    prob = problem(pert=pert, pert_amp=1e-3)
    return dict(name="large", network=NET2, steps=steps,
                instances=[instance(n, boxes_from_sizes(*sizes), bc=1, prob=prob)])


def reference(scale: int = 1, steps: int = 10, max_box: int = 64):
    n = 128 // scale
    prob = problem(ambient_from_T=0, dens_ambient=1e4, p_ambient=1e21, exp_energy=1e52, r_init=1.25e8,
                   X=[1.0], T_init=1e9)
    return dict(name="reference", network=NET13, steps=steps,
                instances=[instance(n, uniform_boxes(n, max(4, max_box // scale)), bc=0, length=1e9, prob=prob)])


WORKLOADS = dict(sedov64=sedov64, sedov128_pert=sedov128_pert, batched=batched, adjoint64=adjoint64, large=large,
                 reference=reference)


def zones(cfg) -> int:
    return sum(int(math.prod(h - l + 1 for l, h in zip(i["dom_lo"], i["dom_hi"]))) for i in cfg["instances"])


def nvar(cfg) -> int:
    return 7 + len(cfg["network"][0])
