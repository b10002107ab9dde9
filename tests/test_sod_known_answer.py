"""Sod shock tube known-answer test of the hydro scheme (CPU, the oracle).

A planar Riemann problem along x in a 128 x 4 x 4 zone box of 1 cm
(rho 1 | 0.125 g/cc, p 1e13 | 1e12 erg/cc, at rest, outflow boundaries): a
left-moving rarefaction, a contact and a right-moving shock, compared with the
exact solution of the ideal-gas Riemann problem (riemann_exact.py, gamma = 5/3:
ions plus the analytic table's non-degenerate electrons at ~1.5e5 K, radiation
below 1e-6 of the pressure; the reference's normalize_species, which stores X
in the rho X slots, changes the gas's mean molecular weight away from
rho = 1 but not p = (2/3) rho e).  With the interface pressure in the momentum
flux (oracle_set_momentum_flux_pressure(1), full Castro's Cartesian form) the
density profile matches the exact one to 0.7% in relative L1 at t = 2.5e-8 s
(bound 2%); with the reference's flux (no pressure in the momentum flux) the
waves do not form and the error is 14 times larger (9.8%).
"""
from __future__ import annotations

import numpy as np

import riemann_exact as RX

GAMMA = 5.0 / 3.0
LEFT = (1.0, 0.0, 1e13)
RIGHT = (0.125, 0.0, 1e12)
T_END = 2.5e-8
NX = 128


def sod_state(nvar, nspec_x=(0.5, 0.5), nx=NX, ny=4):
    """The initial state as a Fortran-order (nx, ny, ny, nvar) array."""
    U = np.zeros((nx, ny, ny, nvar), order="F")
    for i in range(nx):
        rho, u, p = LEFT if i < nx // 2 else RIGHT
        e = p / ((GAMMA - 1.0) * rho)
        U[i, ..., 0] = rho
        U[i, ..., 4] = rho * e
        U[i, ..., 5] = rho * e
        U[i, ..., 6] = 1e5                    # the first EOS solve's starting guess
        for k, x in enumerate(nspec_x):
            U[i, ..., 7 + k] = rho * x
    return U


def sod_domain(nx=NX, ny=4):
    dx = 1.0 / nx
    return dict(boxes=[((0, 0, 0), (nx - 1, ny - 1, ny - 1))], dom_lo=(0, 0, 0), dom_hi=(nx - 1, ny - 1, ny - 1),
                problo=(0.0, 0.0, 0.0), probhi=(1.0, ny * dx, ny * dx), bc=1)


def exact_density(t, nx=NX):
    x = (np.arange(nx) + 0.5) / nx
    return RX.sample(LEFT, RIGHT, GAMMA, (x - 0.5) / t)[:, 0]


def l1_error(rho, t):
    ex = exact_density(t, len(rho))
    return float(np.abs(rho - ex).sum() / ex.sum())


def _run_oracle(pkg, oracle, table, mom_flux_p):
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z, "fast")
    oracle.eos_init(table, "fast")
    oracle.set_momentum_flux_pressure(mom_flux_p, "fast")
    try:
        D = sod_domain()
        lev = oracle.Level(D["boxes"], D["dom_lo"], D["dom_hi"], D["problo"], D["probhi"], D["bc"], 9, variant="fast")
        lev.state(0)[...] = sod_state(9)
        for _ in range(2000):
            if lev.time >= T_END * (1 - 1e-12):
                break
            lev.coarse_step(T_END)
        U = lev.state(0)
        return lev.time, U[:, :, :, 0].mean(axis=(1, 2))
    finally:
        oracle.set_momentum_flux_pressure(False, "fast")


def test_sod_with_pressure_in_the_momentum_flux(pkg, oracle, table):
    t, rho = _run_oracle(pkg, oracle, table, True)
    assert abs(t / T_END - 1) < 1e-12
    err = l1_error(rho, t)
    print("Sod L1(rho) with the pressure in the momentum flux:", err)
    assert err < 0.02


def test_sod_reference_flux(pkg, oracle, table):
    t, rho = _run_oracle(pkg, oracle, table, False)
    err = l1_error(rho, t)
    print("Sod L1(rho) with the reference's flux:", err)
    assert err > 0.05
