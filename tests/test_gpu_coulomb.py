"""Coulomb corrections in the EOS on the GPU (castro_set_coulomb_corrections).

Off by default, as in the reference's eos.F90; its 2017 runs had them on
(scaling/summitdev_20171020/1.out:14).  With the option in both the library
and the oracle (oracle_set_coulomb_corrections, checked against physics in
test_coulomb_cpu.py):

* the exact build follows the oracle through whole coarse steps in every step
  path with the strict per-zone criterion of the configuration tests, and the
  production build likewise (the corrections' cube root and power come from
  CUDA's and the host's libm, which agree to an ulp, not bit for bit: the
  exact build is held to the same per-zone bar as the production build here,
  and to bit-for-bit equality everywhere the option is off);
* the option changes the state (the configurations' ambient gas at 1 g/cc and
  1e6 K has a coupling parameter of ~1.5) and switching it off restores the
  default bit for bit;
* the adjoint, whose EOS has no corrections, refuses to run with it.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_harness import RTOL_L1, assert_strict, cancellation_mask, noise_mask, rel_l1

pytestmark = pytest.mark.gpu


@pytest.fixture()
def coulomb(pkg, oracle):
    libs = [pkg.castro.load(False), pkg.castro.load(True)]
    for L in libs:
        L.castro_set_coulomb_corrections(1)
    for v in ("parity", "fast"):
        oracle.set_coulomb_corrections(True, v)
    yield libs
    for L in libs:
        L.castro_set_coulomb_corrections(0)
    for v in ("parity", "fast"):
        oracle.set_coulomb_corrections(False, v)


def _cfg(pkg):
    return pkg.configs.sedov128_pert(scale=4, max_box=64)      # 32^3 in 8 boxes of 16^3, perturbed


def _levels(oracle, pkg, table, cfg, variant):
    A, Z = cfg["network"]
    oracle.network_init(A, Z, variant)
    oracle.eos_init(table, variant)
    inst = cfg["instances"][0]
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg), variant)
    return lev, inst


@pytest.mark.parametrize("mode", [1, 2, 3, 0], ids=["batched", "plain_box", "persistent", "plain"])
def test_coulomb_steps_match_oracle(pkg, table, oracle, coulomb, mode):
    cfg = _cfg(pkg)
    A, Z = cfg["network"]
    lev, inst = _levels(oracle, pkg, table, cfg, "parity")
    fast, _ = _levels(oracle, pkg, table, cfg, "fast")
    G0 = oracle.assemble(lev, inst)
    sims = {}
    for exact in (True, False):
        L = pkg.castro.init(A, Z, table, exact=exact)
        assert L.castro_coulomb_corrections() == 1
        sims[exact] = pkg.make_sim(L, cfg, mode)
        sims[exact].init_data()
    dx = (inst["probhi"][0] - inst["problo"][0]) / (inst["dom_hi"][0] - inst["dom_lo"][0] + 1)
    steps = 4
    for s in range(steps):
        dto = lev.coarse_step(-1.0)
        fast.coarse_step(-1.0)
        Go = oracle.assemble(lev, inst)
        for exact, sim in sims.items():
            sim.step(1)
            assert abs(sim.dt(0) / dto - 1.0) <= 1e-14, (exact, s, sim.dt(0), dto)
            G = pkg.castro.assemble(inst, sim.box_states()[0])
            if s == 0:
                noise = noise_mask(Go, oracle.assemble(fast, inst)) | cancellation_mask(G0, Go, dto, dx)
                assert_strict(G, Go, noise, what=f"coulomb, mode {mode}, exact={exact}, step 1")
            if s == steps - 1:
                assert float(rel_l1(G, Go).max()) <= RTOL_L1
    for sim in sims.values():
        assert sim.eos_failures() == 0
        sim.close()
    # the option changes the answer
    oracle.set_coulomb_corrections(False)
    ref, _ = _levels(oracle, pkg, table, cfg, "parity")
    for _ in range(steps):
        ref.coarse_step(-1.0)
    R = oracle.assemble(ref, inst)
    rel = np.abs(R - Go) / np.abs(Go).clip(1e-300)
    assert rel[..., 5].max() > 0.1 and rel[..., 0].max() > 0.0    # the ambient rho e, ~12%
    oracle.set_coulomb_corrections(True)


def test_switching_off_restores_the_default(pkg, table, oracle):
    cfg = _cfg(pkg)
    A, Z = cfg["network"]
    inst = cfg["instances"][0]
    out = []
    L = pkg.castro.init(A, Z, table, exact=True)
    for on in (0, 1, 0):
        L.castro_set_coulomb_corrections(on)
        sim = pkg.make_sim(L, cfg, pkg.castro.MODE_BATCHED)
        sim.init_data()
        sim.step(2)
        out.append(pkg.castro.assemble(inst, sim.box_states()[0]))
        sim.close()
    L.castro_set_coulomb_corrections(0)
    assert np.array_equal(out[0], out[2]) and not np.array_equal(out[0], out[1])
    oracle.network_init(A, Z)
    oracle.eos_init(table)
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    lev.coarse_step(-1.0)
    lev.coarse_step(-1.0)
    np.testing.assert_array_equal(out[0], oracle.assemble(lev, inst))


def test_adjoint_refuses_coulomb(pkg, table, coulomb):
    cfg = pkg.configs.adjoint64(scale=4, steps=2)
    L = pkg.castro.init(*cfg["network"], table, exact=False)
    with pytest.raises(pkg.castro.CastroError, match="Coulomb"):
        pkg.adjoint.SedovAdjoint(L, cfg["instances"][0], 2, checkpoint=1)
    L.castro_clear_error()
