"""CPU tests of the oracle (the checker): internal-consistency pins of the EOS,
conservation, symmetry and the committed golden vectors.

The reference ships no golden vectors and cannot be built here (no Fortran
compiler, no AMReX), so parity with the reference itself is unpinned; these
tests pin the oracle against the physics the reference encodes.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

H, AVO, KERG, ME = 6.6260689633e-27, 6.0221417930e23, 1.380650424e-16, 9.1093826e-28
ASOL = 4.0 * 5.67051e-5 / 2.99792458e10


@pytest.fixture(scope="module")
def net2(oracle, table, pkg):
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    return oracle


def analytic_eos(rho, T, abar, zbar):
    """Radiation + ideal ions + the non-degenerate electron gas of the table."""
    ye = zbar / abar
    p = ASOL / 3 * T ** 4 + KERG * AVO / abar * rho * T + KERG * AVO * ye * rho * T
    e = ASOL * T ** 4 / rho + 1.5 * KERG * AVO / abar * T + 1.5 * KERG * AVO * ye * T
    return p, e


def test_table_grid_and_node_exactness(net2, pkg):
    # at table nodes the biquintic interpolation returns the node values, so
    # the EOS must equal the analytic sum of its three components
    d, t = pkg.helm_table.grid()
    abar, zbar = 6.4, 3.2
    ye = zbar / abar
    for j in (10, 60, 120, 199):
        for i in (100, 240, 400):
            T = t[j]
            rho = d[i] / ye
            st = net2.eos(net2.EOS_INPUT_RT, rho=rho, T=T, abar=abar, zbar=zbar)
            p, e = analytic_eos(rho, T, abar, zbar)
            assert st.p == pytest.approx(p, rel=2e-13)
            assert st.e == pytest.approx(e, rel=2e-13)


def test_eos_between_nodes_is_smooth(net2):
    # off-node, the quintic Hermite interpolation of a smooth table is accurate
    abar, zbar = 6.4, 3.2
    for rho, T in [(1.0, 1.7e6), (3.3e2, 4.4e8), (1e5, 2.5e9)]:
        st = net2.eos(net2.EOS_INPUT_RT, rho=rho, T=T, abar=abar, zbar=zbar)
        p, e = analytic_eos(rho, T, abar, zbar)
        assert st.p == pytest.approx(p, rel=1e-6)
        assert st.e == pytest.approx(e, rel=1e-6)
        # gamma_1 of an ideal gas + radiation mixture lies in [4/3, 5/3]
        assert 4.0 / 3.0 - 1e-6 <= st.gam1 <= 5.0 / 3.0 + 1e-6
        assert st.cs == pytest.approx(np.sqrt(st.gam1 * st.p / rho), rel=1e-15)


@pytest.mark.parametrize("T", [2e3, 1e6, 3.7e8, 8e12])
def test_eos_round_trips(net2, T):
    abar, zbar = 6.4, 3.2
    for rho in (1e-6, 1.0, 1e4):
        st = net2.eos(net2.EOS_INPUT_RT, rho=rho, T=T, abar=abar, zbar=zbar)
        re = net2.eos(net2.EOS_INPUT_RE, rho=rho, T=T * 3.0, e=st.e, abar=abar, zbar=zbar)
        assert re.T == pytest.approx(T, rel=1e-8)
        assert re.e == st.e  # input restored exactly (eos.F90:566-568)
        rp = net2.eos(net2.EOS_INPUT_RP, rho=rho, T=T / 5.0, p=st.p, abar=abar, zbar=zbar)
        assert rp.T == pytest.approx(T, rel=1e-8)
        assert rp.p == st.p


def test_eos_newton_floor(net2):
    # T never drops below mintemp = 1e3 (eos.F90:543)
    st = net2.eos(net2.EOS_INPUT_RE, rho=1.0, T=1e4, e=1.0, abar=6.4, zbar=3.2)
    assert st.T >= 1e3


def small_level(oracle, pkg, cfg, inst=0):
    nv = pkg.configs.nvar(cfg)
    return oracle.level_from_instance(cfg["instances"][inst], nv)


def test_periodic_conservation_and_symmetry(oracle, table, pkg):
    cfg = pkg.configs.reference(scale=8, steps=4, max_box=8)   # 16^3 in eight 8^3 boxes, 13 species
    A, Z = cfg["network"]
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    inst = cfg["instances"][0]
    lev, prob = small_level(oracle, pkg, cfg)
    G0 = oracle.assemble(lev, inst)
    for _ in range(cfg["steps"]):
        lev.coarse_step(-1.0)
    G = oracle.assemble(lev, inst)
    assert np.isfinite(G).all()
    # mass and total energy conserved to round-off with periodic boundaries
    assert abs(G[..., 0].sum() / G0[..., 0].sum() - 1) < 1e-13
    assert abs(G[..., 4].sum() / G0[..., 4].sum() - 1) < 1e-13
    # the x<->y transposition maps the problem onto itself
    rho = G[..., 0]
    assert np.abs(rho - rho.transpose(1, 0, 2)).max() <= 1e-14 * rho.max()
    mx, my = G[..., 1], G[..., 2]
    assert np.abs(mx - my.transpose(1, 0, 2)).max() <= 1e-12 * np.abs(mx).max()


def test_outflow_config_runs_and_is_finite(oracle, table, pkg):
    cfg = pkg.configs.sedov64(scale=4, steps=3)
    A, Z = cfg["network"]
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    lev, prob = small_level(oracle, pkg, cfg)
    dts = [lev.coarse_step(-1.0) for _ in range(3)]
    # dt grows by at most 1.1x per step (Source/Castro.cpp:237,264-267)
    assert dts[1] <= 1.1 * dts[0] * (1 + 1e-15) and dts[2] <= 1.1 * dts[1] * (1 + 1e-15)
    G = oracle.assemble(lev, cfg["instances"][0])
    assert np.isfinite(G).all()
    assert (G[..., 0] > 0).all() and (G[..., 6] >= 1e3).all()


def test_golden_vectors(oracle, table, pkg):
    """Oracle outputs pinned at commit time (tests/golden/make_golden.py)."""
    path = os.path.join(GOLDEN, "oracle_golden.json")
    with open(path) as fp:
        gold = json.load(fp)
    from golden_cases import compute_cases  # noqa: E402

    cur = compute_cases(oracle, pkg, table)
    assert set(cur) == set(gold)
    for k, v in gold.items():
        np.testing.assert_allclose(np.asarray(cur[k]), np.asarray(v), rtol=1e-14, atol=0, err_msg=k)
