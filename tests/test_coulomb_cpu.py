"""Coulomb corrections of the EOS on the oracle (CPU): an option, off by
default as in the reference's eos.F90; the reference's 2017 runs had them on
(scaling/summitdev_20171020/1.out:14, "using Coulomb corrections").

Checked against physics rather than against a restatement of the same fits:
the coupling parameter Gamma computed here from its definition, the
Debye-Hueckel limit at weak coupling, continuity of the two fits at Gamma = 1,
thermodynamic consistency of the whole EOS with the corrections on (the
analytic derivatives against central differences, the Maxwell relation
de/drho|T = (p - T dp/dT) / rho^2 and dS/dT = (de/dT) / T), and the default
path bit for bit unchanged.
"""
from __future__ import annotations

import math

import pytest

import oracle as O

AVO, KERG, QE = 6.0221417930e23, 1.380650424e-16, 4.80320427e-10
A, Z = (4.0, 16.0), (2.0, 8.0)
X = (0.5, 0.5)
ABAR = 1.0 / sum(x / a for x, a in zip(X, A))
ZBAR = ABAR * sum(x * z / a for x, z, a in zip(X, Z, A))


def gamma(rho, T, abar=ABAR, zbar=ZBAR):
    n_i = AVO * rho / abar
    a = (3.0 / (4.0 * math.pi * n_i)) ** (1.0 / 3.0)
    return zbar * zbar * QE * QE / (a * KERG * T)


def T_for_gamma(rho, g):
    return gamma(rho, 1.0) / g


@pytest.fixture
def coul(pkg, table):
    O.network_init(A, Z)
    O.eos_init(table)
    O.set_coulomb_corrections(True)
    yield
    O.set_coulomb_corrections(False)


def _rt(rho, T):
    return O.eos(O.EOS_INPUT_RT, rho=rho, T=T, abar=ABAR, zbar=ZBAR)


def _off_on(rho, T):
    O.set_coulomb_corrections(False)
    off = _rt(rho, T)
    O.set_coulomb_corrections(True)
    return off, _rt(rho, T)


def test_debye_hueckel_limit(coul):
    """At weak coupling the excess pressure is -Gamma^(3/2) / (2 sqrt 3) of the ion pressure."""
    for rho, g in ((1e-2, 1e-4), (1.0, 1e-3), (1e3, 1e-2)):
        T = T_for_gamma(rho, g)
        off, on = _off_on(rho, T)
        pion = AVO * KERG * rho * T / ABAR
        ratio = (on.p - off.p) / pion
        dh = -g ** 1.5 / (2.0 * math.sqrt(3.0))
        # the fit's next term, a2 Gamma^b2 / 3, is ~0.1 Gamma^2
        assert abs(ratio / dh - 1.0) < 1.2 * g ** 0.49, (rho, g, ratio, dh)


@pytest.mark.parametrize("rho,g", [(1e-3, 1e-3), (1.0, 0.3), (1.0, 1.6), (1e2, 5.0)])
def test_virial_pressure(coul, rho, g):
    """The excess pressure of a Coulomb system is a third of its excess energy density."""
    T = T_for_gamma(rho, g)
    off, on = _off_on(rho, T)
    pc, ec = on.p - off.p, on.e - off.e
    assert pc < 0 and ec < 0
    assert abs(pc / (rho * ec / 3.0) - 1.0) < 1e-9 * abs(on.p / pc)


def test_dropped_where_the_totals_would_turn_negative(coul):
    """With the table's ideal electrons a strongly coupled state (Gamma = 160) would get a
    negative total energy: the correction is not applied there."""
    rho = 1e6
    T = T_for_gamma(rho, 160.0)
    off, on = _off_on(rho, T)
    assert (on.p, on.e, on.dpdT, on.dedT) == (off.p, off.e, off.dpdT, off.dedT)


def test_fits_meet_at_gamma_one(coul):
    rho = 10.0
    T1 = T_for_gamma(rho, 1.0)
    lo, hi = _rt(rho, T1 * (1 + 1e-9)), _rt(rho, T1 * (1 - 1e-9))        # Gamma just below / above 1
    O.set_coulomb_corrections(False)
    base = _rt(rho, T1)
    O.set_coulomb_corrections(True)
    ec_lo, ec_hi = lo.e - base.e, hi.e - base.e
    assert abs(ec_lo / ec_hi - 1.0) < 2e-5


STATES = [(1e-3, 1e-3), (1.0, 0.3), (1.0, 1.6), (1e2, 3.0), (1e2, 5.0)]   # (rho, Gamma)
FIELDS = ("p", "e", "s", "dpdT", "dpdr", "dedT", "dedr", "dsdT")


def _coulomb_part(rho, T):
    """The corrections' own contribution: the EOS with them on minus off (the table's part
    is the same in both; its dp/drho, from the separate dpdf table, is consistent with p
    only to ~3e-6)."""
    off, on = _off_on(rho, T)
    c = {f: getattr(on, f) - getattr(off, f) for f in FIELDS}
    c.update({"total_" + f: getattr(on, f) for f in FIELDS})
    return c


@pytest.mark.parametrize("rho,g", STATES)
def test_derivatives_against_differences(coul, rho, g):
    T = T_for_gamma(rho, g)
    c = _coulomb_part(rho, T)
    h = 1e-5
    for var, dp, de, ds in (("T", c["dpdT"], c["dedT"], c["dsdT"]), ("rho", c["dpdr"], c["dedr"], None)):
        if var == "T":
            a, b, step = _coulomb_part(rho, T * (1 + h)), _coulomb_part(rho, T * (1 - h)), 2 * h * T
        else:
            a, b, step = _coulomb_part(rho * (1 + h), T), _coulomb_part(rho * (1 - h), T), 2 * h * rho
        for f, d in (("p", dp), ("e", de), ("s", ds)):
            if d is None:
                continue
            fd = (a[f] - b[f]) / step
            # the on-minus-off difference cancels the total's leading digits: rounding of the
            # total, over the step, bounds what the difference can resolve
            noise = 1e-15 * abs(a["total_" + f]) / step
            assert abs(fd - d) <= 1e-7 * abs(d) + 10 * noise, (var, f, fd, d)


@pytest.mark.parametrize("rho,g", STATES)
def test_maxwell_relations(coul, rho, g):
    """de/drho|T = (p - T dp/dT) / rho^2 and dS/dT = (de/dT) / T for the corrections."""
    T = T_for_gamma(rho, g)
    c = _coulomb_part(rho, T)
    maxwell = (c["p"] - T * c["dpdT"]) / (rho * rho)
    scale = 1e-13 * (abs(c["total_p"]) + abs(T * c["total_dpdT"]) + abs(rho * rho * c["total_dedr"]))
    assert abs(c["dedr"] - maxwell) <= 1e-10 * abs(c["p"] / (rho * rho)) + scale / (rho * rho)
    assert abs(c["dsdT"] - c["dedT"] / T) <= 1e-10 * abs(c["dedT"] / T) + 1e-13 * abs(c["total_dedT"] / T)


def test_off_by_default_and_unchanged(pkg, table):
    O.network_init(A, Z)
    O.eos_init(table)
    ref = _rt(1.0, 1e6)
    O.set_coulomb_corrections(True)
    on = _rt(1.0, 1e6)
    O.set_coulomb_corrections(False)
    again = _rt(1.0, 1e6)
    assert (again.p, again.e, again.gam1, again.cs) == (ref.p, ref.e, ref.gam1, ref.cs)
    assert on.p < ref.p                                   # Gamma ~ 1.5 in the configurations' ambient gas
    assert 1.0 < gamma(1.0, 1e6) < 2.0
