"""The smooth-advection known answer (test_advection_known_answer.py) on the GPU.

The reference's own scheme, the library's default: the production build
carries the density wave to the translated profile with the relative L1
error the oracle measures (7.9e-4 at 64^3, bound 1.2e-3), and the exact build
matches the oracle (parity build) bit for bit on the uploaded 32^3 state.
"""
from __future__ import annotations

import numpy as np
import pytest

import test_advection_known_answer as ADV

pytestmark = pytest.mark.gpu


def _gpu(pkg, table, n, exact, mode):
    C = pkg.configs
    inst = dict(ADV.advection_domain(n), problem=C.problem(r_init=0.1), n=n, stop_time=ADV.T_END)
    cfg = dict(name="advection", network=C.NET2, steps=0, instances=[inst])
    L = pkg.castro.init(*C.NET2, table, exact=exact)
    assert L.castro_momentum_flux_pressure() == 0          # the reference's flux
    sim = pkg.make_sim(L, cfg, mode)
    sim.upload(ADV.advection_state(n).ravel(order="F"))
    dts = []
    while sim.time(0) < ADV.T_END * (1 - 1e-12):
        sim.step(1)
        dts.append(sim.dt(0))
    G = pkg.castro.assemble(inst, sim.box_states()[0])
    t = sim.time(0)
    sim.close()
    return t, G, dts


def test_advection_gpu_error(pkg, table):
    t, G, _ = _gpu(pkg, table, 64, False, pkg.castro.MODE_BATCHED)
    err = ADV.l1_error(G[..., 0], 64, t)
    print("GPU advection L1(rho), 64^3:", err)
    assert err < 1.2e-3


@pytest.mark.parametrize("mode", [1, 2], ids=["batched", "plain_box"])
def test_advection_exact_matches_oracle(pkg, table, oracle, mode):
    n = 32
    t, G, dts = _gpu(pkg, table, n, True, mode)
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    D = ADV.advection_domain(n)
    lev = oracle.Level(D["boxes"], D["dom_lo"], D["dom_hi"], D["problo"], D["probhi"], D["bc"], 9)
    lev.state(0)[...] = ADV.advection_state(n)
    dto = []
    while lev.time < ADV.T_END * (1 - 1e-12):
        dto.append(lev.coarse_step(ADV.T_END))
    np.testing.assert_array_equal(G, lev.state(0))
    assert dts == dto
