"""The Fermi-Dirac Helmholtz table (mini-castro_b200/helm_fd.py) on the CPU.

* the generalized Fermi-Dirac integrals against their closed forms and
  asymptotic series, and their eta / beta partials against differences;
* thermodynamic consistency of the tabulated quantities over the grid:
  f_T = -s, the Maxwell relation ds/dd = -P_T / d^2, f_TT = -s_T, and
  e = f + T s equal to the kinetic plus pair rest-mass energy;
* the physical limits: ideal non-degenerate gas, the T = 0 Chandrasekhar
  pressure, and the ultra-relativistic pair plasma (7/4 of radiation's 1/3 a T^4);
* the oracle's EOS (Newton inversion included) on a table whose window around
  a Sedov ambient state is computed by the generator.
"""
from __future__ import annotations

import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def H(pkg):
    return pkg.helm_fd


def test_fd_integrals_closed_forms(H):
    F = H.fd_partials(np.array([0.0, -30.0, 1e4]), np.zeros(3))
    zeta32 = 2.612375348685488
    assert abs(F[0][0][0][0] / ((1 - 2 ** -0.5) * math.gamma(1.5) * zeta32) - 1) < 1e-14
    # non-degenerate: Gamma(3/2) (e^eta - e^(2 eta) / 2^(3/2))
    nd = math.gamma(1.5) * (math.exp(-30.0) - math.exp(-60.0) / 2 ** 1.5)
    assert abs(F[0][0][0][1] / nd - 1) < 1e-14
    # degenerate: Sommerfeld, eta^(3/2) / (3/2) + pi^2 / 6 * (1/2) eta^(-1/2)
    eta = 1e4
    assert abs(F[0][0][0][2] / (eta ** 1.5 / 1.5 + math.pi ** 2 / 12 * eta ** -0.5) - 1) < 1e-14


@pytest.mark.parametrize("eta,beta", [(-5.0, 1e-3), (3.0, 0.5), (80.0, 2.0), (400.0, 1e-4)])
def test_fd_partials_match_differences(H, eta, beta):
    F = H.fd_partials(np.array([eta]), np.array([beta]))
    h_e, h_b = 1e-4 * max(1.0, abs(eta)), 1e-4 * beta
    Fe = [H.fd_partials(np.array([eta + s * h_e]), np.array([beta])) for s in (-1, 1)]
    Fb = [H.fd_partials(np.array([eta]), np.array([beta + s * h_b])) for s in (-1, 1)]
    for k in range(3):
        for a in range(3):
            for b in range(3 - a):
                de = (Fe[1][k][a][b][0] - Fe[0][k][a][b][0]) / (2 * h_e)
                db = (Fb[1][k][a][b][0] - Fb[0][k][a][b][0]) / (2 * h_b)
                assert abs(de - F[k][a + 1][b][0]) <= 1e-6 * (abs(F[k][a + 1][b][0]) + abs(F[k][a][b][0]) * 1e-3)
                assert abs(db - F[k][a][b + 1][0]) <= 1e-6 * (abs(F[k][a][b + 1][0]) + abs(F[k][a][b][0]) * 1e-3)


def _consistency(H, d, T):
    vals, jets = H.node_values(d, np.full_like(d, T))
    s, P, psi, E, npos = jets["s_jet"], jets["P_jet"], jets["psi_jet"], jets["E_jet"], jets["npos_jet"]
    u, v = H._jet_vars((d.size,))
    inv_d = H._jet_fun(u + d, [1 / d, -1 / d ** 2, 2 / d ** 3, -6 / d ** 4])
    f = (H.AVO * H.MEC2) * psi - P * inv_d
    e = (E.deriv(0, 0) + 2 * H.MEC2 * npos.deriv(0, 0)) / d
    err = {
        "f_T = -s": np.abs(f.deriv(0, 1) + s.deriv(0, 0)) / np.abs(s.deriv(0, 0)),
        "f_TT = -s_T": np.abs(f.deriv(0, 2) + s.deriv(0, 1)) / np.abs(s.deriv(0, 1)),
        "s_d = -P_T/d^2": np.abs(s.deriv(1, 0) + P.deriv(0, 1) / d ** 2) / np.abs(P.deriv(0, 1) / d ** 2),
        "e = f + Ts": np.abs(vals[0][0] + T * s.deriv(0, 0) - e) / np.abs(e),
        "table fd = f_d": np.abs(vals[0][1] - f.deriv(1, 0)) / np.abs(vals[0][1]),
    }
    return vals, err


@pytest.mark.parametrize("jT", [0, 60, 100, 140, 200])
def test_thermodynamic_consistency(H, pkg, jT):
    d1, t1 = pkg.helm_table.grid()
    d = d1[::45]
    vals, err = _consistency(H, d, t1[jT])
    eta = vals[2][0]
    # the thermal derivatives of the degenerate bulk are Fermi-surface integrals
    # whose odd part cancels: relative rounding ~ eps * eta
    bound = np.maximum(1e-11, 3e-16 * np.abs(eta) * 100)
    for name, e in err.items():
        assert (e <= bound).all(), f"T={t1[jT]:.1e}: {name}: worst {e.max():.2e} at d={d[np.argmax(e / bound)]:.1e}"


def test_limits(H):
    k, h, c, me, avo = H.KERG, H.H_PLANCK, H.CLIGHT, H.ME, H.AVO
    # ideal non-degenerate gas: P = N_A k T d to O(beta, e^eta)
    d = np.array([1e-6])
    _, jets = H.node_values(d, np.array([1e5]))
    assert abs(jets["P_jet"].deriv(0, 0)[0] / (avo * k * 1e5 * d[0]) - 1) < 1e-4
    # T -> 0: Chandrasekhar's P(x_F), x_F = p_F / (m_e c)
    d = np.array([1e2, 1e5, 1e8, 1e11])
    _, jets = H.node_values(d, np.full_like(d, 1e3))
    x = h * (3 * avo * d / (8 * math.pi)) ** (1 / 3) / (me * c)
    pch = math.pi * me ** 4 * c ** 5 / (3 * h ** 3) * (x * (2 * x * x - 3) * np.sqrt(1 + x * x) + 3 * np.arcsinh(x))
    assert np.all(np.abs(jets["P_jet"].deriv(0, 0) / pch - 1) < 1e-6)
    # ultra-relativistic pairs at low net density: 7/4 of radiation's a T^4 / 3
    T = 1e13
    _, jets = H.node_values(np.array([1e-12]), np.array([T]))
    a = 8 * math.pi ** 5 * k ** 4 / (15 * h ** 3 * c ** 3)
    assert abs(jets["P_jet"].deriv(0, 0)[0] / (7.0 / 4.0 * a * T ** 4 / 3) - 1) < 1e-5


def test_oracle_eos_on_fd_window(H, pkg, tmp_path, oracle):
    """The oracle's EOS (eos.F90 restated) on a table whose window around the
    Sedov ambient (rho = 1, Ye = 1/2, T = 1e6..1e8) holds the Fermi-Dirac
    values: the tabulated pressure is reproduced at the nodes, the EOS_RE
    Newton inversion recovers T, and the thermodynamic derivatives are sane."""
    d1, t1 = pkg.helm_table.grid()
    rows = range(58, 104)             # T = 10^5.9 .. 10^8.15
    cols = range(226, 250)            # d = 10^-0.7 .. 10^0.45
    path = str(tmp_path / "helm_fd_window.dat")
    H.write_table(path, workers=1, rows=rows, cols=cols)
    A, Z = pkg.configs.NET2
    oracle.network_init(A, Z)
    oracle.eos_init(path)
    abar = 1.0 / (0.5 / A[0] + 0.5 / A[1])
    zbar = abar * (0.5 * Z[0] / A[0] + 0.5 * Z[1] / A[1])
    ye = zbar / abar
    # at a node, the electron pressure is the tabulated d^2 f_d
    j, i = 80, 240
    rho = d1[i] / ye
    st = oracle.eos(1, rho=rho, T=t1[j], abar=abar, zbar=zbar)
    vals, _ = H.node_values(np.array([d1[i]]), np.array([t1[j]]))
    pe = d1[i] ** 2 * vals[0][1][0]
    prad = 7.5657e-15 * t1[j] ** 4 / 3
    pion = H.AVO * H.KERG * rho * t1[j] / abar
    assert abs((st.p - prad - pion) / pe - 1) < 1e-3   # radiation constant of the EOS vs the rounded one here
    for T in (1.3e6, 7.7e6, 4.1e7):
        for rho in (0.5, 1.0, 2.0):
            st = oracle.eos(1, rho=rho, T=T, abar=abar, zbar=zbar)
            assert st.p > 0 and st.e > 0 and st.cv > 0 and 1.0 < st.gam1 < 5.0 / 3.0 + 1e-9
            back = oracle.eos(2, rho=rho, T=0.5 * T, e=st.e, abar=abar, zbar=zbar)
            assert abs(back.T / T - 1) < 1e-8
