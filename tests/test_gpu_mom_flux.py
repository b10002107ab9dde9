"""The interface pressure in the normal momentum flux (castro_set_momentum_flux_pressure).

The reference's compute_flux carries rho u u alone in the normal momentum flux
(Source/riemann.F90:306-308), so its blasts expand far slower than the
Sedov-Taylor solution; the library's default reproduces that.  With the option
the flux is rho u u + p, full Castro's Cartesian form, and the same kernels
follow Sedov-Taylor.  Here, on the GPU:

* the exact build with the option matches the oracle with its counterpart
  option (oracle_set_momentum_flux_pressure) bit for bit, in the per-routine,
  drop-in, batched and persistent paths;
* the production build with the option follows R(t) = 1.1517 (E t^2/rho)^(1/5)
  (gamma = 5/3) to 3% on a 64^3 blast (see test_sedov_known_answer.py for the
  setup), and without it falls far behind (the reference's behaviour);
* (the adjoint of compute_flux with the option: test_gpu_adjoint.py.)
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XI0 = 1.1517


@pytest.fixture()
def option(pkg, oracle):
    """Switch the option on in both builds of the library and the parity oracle; off afterwards."""
    libs = [pkg.castro.load(False), pkg.castro.load(True)]
    for L in libs:
        L.castro_set_momentum_flux_pressure(1)
    oracle.set_momentum_flux_pressure(True)
    yield libs
    for L in libs:
        L.castro_set_momentum_flux_pressure(0)
    oracle.set_momentum_flux_pressure(False)


@pytest.mark.parametrize("mode", [0, 1, 2, 3], ids=["plain", "batched", "plain_box", "persistent"])
def test_option_matches_oracle_bitwise(pkg, table, oracle, option, mode):
    cfg = pkg.configs.sedov128_pert(scale=4, max_box=64)    # 32^3 in 8 boxes of 16^3, perturbed
    A, Z = cfg["network"]
    steps = 3
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    inst = cfg["instances"][0]
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    dto = [lev.coarse_step(-1.0) for _ in range(steps)]
    Go = oracle.assemble(lev, inst)
    L = pkg.castro.init(A, Z, table, exact=True)
    assert L.castro_momentum_flux_pressure() == 1
    sim = pkg.make_sim(L, cfg, mode)
    sim.init_data()
    dts = []
    for _ in range(steps):
        sim.step(1)
        dts.append(sim.dt(0))
    G = pkg.castro.assemble(inst, sim.box_states()[0])
    sim.close()
    np.testing.assert_array_equal(G, Go)
    assert dts == dto
    # and the option changes the answer: the reference form differs
    oracle.set_momentum_flux_pressure(False)
    lev2, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    for _ in range(steps):
        lev2.coarse_step(-1.0)
    assert not np.array_equal(oracle.assemble(lev2, inst), Go)
    oracle.set_momentum_flux_pressure(True)


def _blast(pkg, table, n, on, r_stop=0.38, max_steps=900):
    C = pkg.configs
    prob = C.problem(dens_ambient=1.0, T_ambient=1e3, exp_energy=1e12, r_init=0.125)   # as the 32^3 CPU test's 4 zones
    cfg = dict(name="sedov_known_answer", network=C.NET2, steps=0,
               instances=[C.instance(n, C.uniform_boxes(n, 32), bc=1, prob=prob)])
    L = pkg.castro.init(*C.NET2, table)
    L.castro_set_momentum_flux_pressure(1 if on else 0)
    try:
        sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
        sim.init_data()
        rows = []
        for s in range(1, max_steps + 1):
            sim.step(1)
            if s % 20 == 0 and s >= 100:
                r = sim.blast_radius()[0]
                t = sim.time(0)
                rows.append((t, r, XI0 * (1e12 * t * t) ** 0.2))
                if r > r_stop:
                    break
        sim.close()
    finally:
        L.castro_set_momentum_flux_pressure(0)
    return rows


def test_sedov_taylor_gpu(pkg, table):
    rows = _blast(pkg, table, 64, True)
    radii = np.array([r for _, r, _ in rows])
    ratios = np.array([r / rs for _, r, rs in rows])
    print("R, R/R_ST:", [(round(r, 3), round(q, 4)) for r, q in zip(radii, ratios)])
    assert radii[-1] > 0.3
    sel = radii > 0.2
    assert sel.any() and np.all(np.abs(ratios[sel] - 1.0) < 0.03), list(zip(radii, ratios))
    ref = _blast(pkg, table, 64, False, max_steps=300)
    assert ref[-1][1] / ref[-1][2] < 0.6, ref


def _sod_gpu(pkg, table, exact, on):
    import test_sod_known_answer as S

    C = pkg.configs
    inst = dict(S.sod_domain(), problem=C.problem(r_init=0.1), n=S.NX, stop_time=S.T_END)
    cfg = dict(name="sod", network=C.NET2, steps=0, instances=[inst])
    L = pkg.castro.init(*C.NET2, table, exact=exact)
    L.castro_set_momentum_flux_pressure(1 if on else 0)
    try:
        sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
        sim.upload(S.sod_state(9).ravel(order="F"))
        dts = []
        for _ in range(2000):
            if sim.time(0) >= S.T_END * (1 - 1e-12):
                break
            sim.step(1)
            dts.append(sim.dt(0))
        G = pkg.castro.assemble(inst, sim.box_states()[0])
        t = sim.time(0)
        sim.close()
    finally:
        L.castro_set_momentum_flux_pressure(0)
    return t, G, dts


def test_sod_gpu(pkg, table, oracle):
    """The Sod shock tube of test_sod_known_answer.py on the GPU, uploaded as the
    initial state: the production build with the option to 2% of the exact
    solution in relative L1, and the exact build with the option bit for bit
    against the oracle (parity build) with its option."""
    import test_sod_known_answer as S

    t, G, _ = _sod_gpu(pkg, table, False, True)
    assert abs(t / S.T_END - 1) < 1e-12
    err = S.l1_error(G[:, :, :, 0].mean(axis=(1, 2)), t)
    print("GPU Sod L1(rho):", err)
    assert err < 0.02
    # exact build against the parity oracle, both with the option
    t, G, dts = _sod_gpu(pkg, table, True, True)
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    oracle.set_momentum_flux_pressure(True)
    try:
        D = S.sod_domain()
        lev = oracle.Level(D["boxes"], D["dom_lo"], D["dom_hi"], D["problo"], D["probhi"], D["bc"], 9)
        lev.state(0)[...] = S.sod_state(9)
        dto = []
        while lev.time < S.T_END * (1 - 1e-12):
            dto.append(lev.coarse_step(S.T_END))
        np.testing.assert_array_equal(G, lev.state(0))
        assert dts == dto
    finally:
        oracle.set_momentum_flux_pressure(False)
