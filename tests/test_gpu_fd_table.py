"""The hydro path on the Fermi-Dirac Helmholtz table (mini-castro_b200/helm_fd.py).

The configurations run on the analytic non-degenerate table; this module runs
the same kernels on the table computed from Fermi-Dirac integrals (electron-
positron gas in pair equilibrium, degenerate and relativistic where the grid
reaches), against the oracle on the same file:

* compute_temp (the EOS_RE Newton inversion) on zones spread log-uniformly over
  1e-4..1e6 g/cc and 1e4..1e10 K;
* 16^3 Sedov runs of 5 steps: the 2-species outflow problem and the reference
  problem's constants (13 species, periodic).

The exact build must match the oracle bit for bit, the production build to the
tolerances of the other kernel and step tests.  The table is generated on
first use (data/helm_table_fd.dat) when it is not already there.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_harness import RTOL_KERNEL, RTOL_STEP, assert_match, from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fd_table(pkg, table, oracle):
    path = pkg.helm_fd.ensure_table()
    yield path
    # the modules after this one expect the library and the oracle on the default table
    for exact in (False, True):
        pkg.castro.init(*pkg.configs.NET2, table, exact=exact)
    oracle.eos_init(table)


def _random_state(oracle, A, Z, n=8, seed=7):
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    rho = 10.0 ** rng.uniform(-4.0, 6.0, shape)
    T = 10.0 ** rng.uniform(4.0, 10.0, shape)
    X = np.array([0.5, 0.5])
    abar = 1.0 / np.sum(X / np.asarray(A))
    zbar = abar * np.sum(X * np.asarray(Z) / np.asarray(A))
    U = np.zeros(shape + (7 + len(A),), order="F")
    for idx in np.ndindex(shape):
        st = oracle.eos(1, rho=rho[idx], T=T[idx], abar=abar, zbar=zbar)
        U[idx + (0,)] = rho[idx]
        U[idx + (4,)] = rho[idx] * st.e
        U[idx + (5,)] = rho[idx] * st.e
        U[idx + (6,)] = 0.6 * T[idx]                 # the Newton iteration's starting guess
        for k in range(len(A)):
            U[idx + (7 + k,)] = rho[idx] * X[k]
    return U, T


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_compute_temp_on_fd_table(pkg, fd_table, oracle, exact):
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(fd_table)
    U, T = _random_state(oracle, A, Z)
    lo, hi = (0, 0, 0), (7, 7, 7)
    ref = np.asfortranarray(U.copy())
    oracle.call("compute_temp", lo, hi, ref, lo, hi)
    assert np.abs(ref[..., 6] / T - 1).max() < 1e-7           # the inversion recovers T
    L = pkg.castro.init(A, Z, fd_table, exact=exact)
    d = to_dev(U)
    pkg.castro.call(L, "compute_temp", lo, hi, d, lo, hi)
    got = from_dev(d)
    assert_match(got, ref, exact, rtol=RTOL_KERNEL, what="compute_temp on the Fermi-Dirac table")


WORKLOADS = {
    "sedov16_outflow": lambda c: c.sedov64(scale=4),                 # 16^3, 2 species, rho 1, T 1e6
    "reference16_periodic": lambda c: c.reference(scale=8, max_box=64),  # 13 species, rho 1e4, p 1e21
}


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
@pytest.mark.parametrize("wl", list(WORKLOADS))
def test_sedov_on_fd_table(pkg, fd_table, oracle, wl, exact):
    cfg = WORKLOADS[wl](pkg.configs)
    A, Z = cfg["network"]
    steps = 5
    oracle.network_init(A, Z)
    oracle.eos_init(fd_table)
    inst = cfg["instances"][0]
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    dto = [lev.coarse_step(-1.0) for _ in range(steps)]
    Go = oracle.assemble(lev, inst)
    L = pkg.castro.init(A, Z, fd_table, exact=exact)
    sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
    sim.init_data()
    dts = []
    for _ in range(steps):
        sim.step(1)
        dts.append(sim.dt(0))
    G = pkg.castro.assemble(inst, sim.box_states()[0])
    assert sim.eos_failures() == 0
    sim.close()
    if exact:
        np.testing.assert_array_equal(G, Go)
        assert dts == dto
    else:
        assert_match(G, Go, False, rtol=RTOL_STEP * 10, what=f"{wl} on the Fermi-Dirac table")
        np.testing.assert_allclose(dts, dto, rtol=1e-14)
