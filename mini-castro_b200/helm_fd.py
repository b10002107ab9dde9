"""Fermi-Dirac electron-positron free-energy table in the layout of ``helm_table.dat``.

``eos_init`` (Source/eos.F90:580-734) reads 541 x 201 nodes of the electron-
positron Helmholtz free energy per unit ``d = rho * Ye`` and its derivatives on
the grid d = 10**(-12 + 0.05 i) g/cc, T = 10**(3 + 0.05 j) K.  The reference
repository does not carry the file, and ``helm_table.py`` writes an analytic
non-degenerate electron gas in its place.  This module computes the table the
file is made of: a relativistic electron-positron gas of arbitrary degeneracy in
pair equilibrium, following the published construction of the Helmholtz EOS
(Timmes & Swesty 2000, ApJS 126, 501; Timmes & Arnett 1999, ApJS 125, 277):

* generalized Fermi-Dirac integrals
  F_k(eta, beta) = int_0^inf x^k sqrt(1 + beta x / 2) / (exp(x - eta) + 1) dx,
  k = 1/2, 3/2, 5/2, with beta = k T / (m_e c^2) and eta the electron
  chemical potential (rest mass excluded) over k T; the positrons'
  eta_+ = -eta - 2 / beta (pair equilibrium);
* number density n = K beta^(3/2) (F_1/2 + beta F_3/2), pressure
  P = (2/3) K m_e c^2 beta^(5/2) (F_3/2 + beta/2 F_5/2), kinetic energy
  density E = K m_e c^2 beta^(5/2) (F_3/2 + beta F_5/2), K = 8 pi sqrt(2)
  (m_e c / h)^3, for electrons (eta) and positrons (eta_+);
* eta(d, T) from charge neutrality n_- - n_+ = N_A d;
* free energy per unit d: f = N_A k T eta - P / d (net electron rest mass
  excluded, pair rest mass included), entropy s = (E_- + E_+ + 2 m_e c^2 n_+
  + P) / (T d) - N_A k eta, so that e = f + T s = (E_- + E_+ + 2 m_e c^2 n_+) / d.

The derivatives the biquintic and bicubic interpolations need are exact
derivatives, not differences: every quantity is carried as a truncated Taylor
polynomial (a jet) in (delta d, delta T) to third order.  The integrals' own
partial derivatives in eta and beta are integrals of the differentiated
integrand, and eta's jet follows from neutrality by Newton iteration on jets.
Table entries:

* f, fd = P/d^2, ft = -s, fdd = P_d/d^2 - 2P/d^3, ftt = -s_T, fdt = P_T/d^2,
  fddt = P_dT/d^2 - 2P_T/d^3, fdtt = P_TT/d^2, fddtt = P_dTT/d^2 - 2P_TT/d^3;
* dpdf = P_d and its d, T and (d,d,T) derivatives: dpdfd = P_dd, dpdft = P_dT,
  dpdfdt = P_ddT;
* ef = eta, efd, eft, efdt;
* xf = n_- + n_+ (electrons and positrons), xfd, xft, xfdt.

Quadrature: per node, Gauss-Legendre in t = sqrt(x) over pieces graded
geometrically toward t = 0 (the beta branch point at t = +-i sqrt(2/beta))
and pieces of width 2 in x across the Fermi surface, the tail beyond
x = max(eta, 0) + 50 dropped (below 1e-16 of the integral).
"""
from __future__ import annotations

import math
import os

import numpy as np

try:
    from . import helm_table as _ht
except ImportError:   # loaded by file path
    import importlib.util as _ilu

    _spec = _ilu.spec_from_file_location("helm_table", os.path.join(os.path.dirname(__file__), "helm_table.py"))
    _ht = _ilu.module_from_spec(_spec)
    _spec.loader.exec_module(_ht)

IMAX, JMAX = _ht.IMAX, _ht.JMAX
H_PLANCK, AVO, KERG, ME = _ht.H_PLANCK, _ht.AVO, _ht.KERG, _ht.ME
CLIGHT = 2.99792458e10
MEC2 = ME * CLIGHT * CLIGHT
KFD = 8.0 * math.pi * math.sqrt(2.0) * (ME * CLIGHT / H_PLANCK) ** 3
KS = (0.5, 1.5, 2.5)
ORDER = 3                      # jets carry derivatives up to third order
TAIL = 50.0                    # x beyond max(eta, 0) + TAIL is dropped
BETA_PAIR = 0.02               # above this beta, neutrality is solved for eta + 1/beta

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "helm_table_fd.dat")

# ---------------------------------------------------------------------------
# quadrature
# ---------------------------------------------------------------------------
_GL = {n: np.polynomial.legendre.leggauss(n) for n in (8, 10)}
N_GEO_A = 30                   # geometric pieces of [0, T_a]
N_GEO_B = 16                   # geometric pieces of the first Fermi-surface piece
N_UNI_B = 49                   # further pieces of width 2 in x


def _gl_piece(lo, hi, n):
    """Gauss-Legendre nodes and weights of n points on per-point intervals [lo, hi]."""
    z, wz = _GL[n]
    h = 0.5 * (hi - lo)
    return (0.5 * (hi + lo))[:, None] + h[:, None] * z[None, :], h[:, None] * wz[None, :]


def _nodes(eta):
    """Quadrature of int_0^inf dx per point: x nodes, y = x - eta, and dx weights, shape (P, Q).

    [0, x_a], x_a = max(eta - TAIL, 0): in t = sqrt(x), pieces graded
    geometrically toward t = 0.  [x_a, max(eta, 0) + TAIL], the Fermi surface:
    N_UNI_B + 1 pieces of equal width, the first graded toward its start; in t
    when x_a = 0 (the x^(1/2) and beta branch points near its start), else in
    y = x - eta, so that y is exact where the Fermi factor varies even when x
    is large (eta up to ~1e10 at the table's coldest, densest corner)."""
    eta = np.asarray(eta, dtype=np.float64)
    xa = np.maximum(eta - TAIL, 0.0)
    xb = np.maximum(eta, 0.0) + TAIL
    ta = np.sqrt(xa)
    deg = eta > TAIL
    X, Y, W = [], [], []

    def add_t(lo, hi, n):
        t, h = _gl_piece(lo, hi, n)
        x = t * t
        X.append(x)
        Y.append(x - eta[:, None])
        W.append(2.0 * t * h)                                    # dx = 2 t dt

    if (ta > 0).any():   # some point is degenerate beyond TAIL
        for m in range(N_GEO_A):
            add_t(ta * 0.5 ** (m + 1), ta * 0.5 ** m, 10)
        add_t(np.zeros_like(ta), ta * 0.5 ** N_GEO_A, 10)
    # the Fermi surface
    wx = (xb - xa) / (N_UNI_B + 1)
    t1 = np.sqrt(xa + wx)
    ylo = np.where(deg, -TAIL, -eta)                             # y at x_a
    bounds = [(1.0 * 0.5 ** (m + 1), 1.0 * 0.5 ** m, 8) for m in range(N_GEO_B)] + [(0.0, 0.5 ** N_GEO_B, 8)]
    for flo, fhi, n in bounds:                                   # first piece, graded toward its start
        tt, ht = _gl_piece(ta + (t1 - ta) * flo, ta + (t1 - ta) * fhi, n)
        yy, hy = _gl_piece(ylo + wx * flo, ylo + wx * fhi, n)
        x_t = tt * tt
        X.append(np.where(deg[:, None], eta[:, None] + yy, x_t))
        Y.append(np.where(deg[:, None], yy, x_t - eta[:, None]))
        W.append(np.where(deg[:, None], hy, 2.0 * tt * ht))
    for m in range(1, N_UNI_B + 1):   # 10 points: the Fermi factor's poles lie pi off the real axis
        tt, ht = _gl_piece(np.sqrt(xa + m * wx), np.sqrt(xa + (m + 1) * wx), 10)
        yy, hy = _gl_piece(ylo + m * wx, ylo + (m + 1) * wx, 10)
        x_t = tt * tt
        X.append(np.where(deg[:, None], eta[:, None] + yy, x_t))
        Y.append(np.where(deg[:, None], yy, x_t - eta[:, None]))
        W.append(np.where(deg[:, None], hy, 2.0 * tt * ht))
    return np.concatenate(X, axis=1), np.concatenate(Y, axis=1), np.concatenate(W, axis=1)


def _fermi_factors(y, amax):
    """d^a/d eta^a of 1/(exp(y) + 1), y = x - eta, a = 0..amax (stable for either sign of y)."""
    e = np.exp(-np.abs(y))
    f = np.where(y > 0, e / (1.0 + e), 1.0 / (1.0 + e))
    g = np.where(y > 0, 1.0 / (1.0 + e), e / (1.0 + e))        # 1 - f
    out = [f]
    if amax >= 1:
        fg = f * g
        out.append(fg)
    if amax >= 2:
        out.append(fg * (g - f))
    if amax >= 3:
        out.append(fg * (1.0 - 6.0 * fg))
    return out, g


def _beta_factors(x, beta, bmax):
    """d^b/d beta^b of sqrt(1 + beta x / 2), b = 0..bmax."""
    s = 1.0 + 0.5 * beta[:, None] * x
    r = np.sqrt(s)
    out = [r]
    if bmax >= 1:
        out.append(0.25 * x / r)
    if bmax >= 2:
        out.append(-x * x / (16.0 * s * r))
    if bmax >= 3:
        out.append(3.0 * x ** 3 / (64.0 * s * s * r))
    return out


def fd_partials(eta, beta, order=ORDER):
    """F[k][a][b] = d^(a+b) F_k / d eta^a d beta^b at each (eta, beta), a + b <= order, k over KS."""
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    beta = np.broadcast_to(np.asarray(beta, dtype=np.float64), eta.shape).copy()
    x, y, w = _nodes(eta)
    fe, _ = _fermi_factors(y, order)
    gb = _beta_factors(x, beta, order)
    sx = np.sqrt(x)
    xk = [sx, sx * x, sx * x * x]
    out = []
    for ki in range(3):
        row = [[None] * (order + 1) for _ in range(order + 1)]
        for a in range(order + 1):
            wa = w * fe[a] * xk[ki]
            for b in range(order + 1 - a):
                row[a][b] = np.sum(wa * gb[b], axis=1)
        out.append(row)
    return out


def _net_density(eta, phi, beta):
    """n_- - n_+ and its derivative in eta, at eta (electrons), eta_+ = -eta - 2/beta
    (positrons), phi = eta + 1/beta given separately so that the difference of
    the two Fermi factors is formed without cancellation when phi is small."""
    etap = -phi - 1.0 / beta
    eref = np.maximum(eta, etap)
    x, y, w = _nodes(eref)
    fm, gm = _fermi_factors(y + (eref - eta)[:, None], 1)
    fp, _ = _fermi_factors(y + (eref - etap)[:, None], 1)
    sx = np.sqrt(x)
    g = np.sqrt(1.0 + 0.5 * beta[:, None] * x)
    base = w * sx * g * (1.0 + beta[:, None] * x)             # x^1/2 g + beta x^3/2 g
    # f_- - f_+ = exp(x - eta) expm1(2 phi) f_- f_+ = expm1(2 phi) f_+ (1 - f_-); the plain
    # difference once the positrons are far below the electrons
    with np.errstate(over="ignore", invalid="ignore"):
        small = (np.abs(phi) < 20.0)[:, None]
        diff = np.where(small, np.expm1(2.0 * np.minimum(phi, 20.0))[:, None] * fp[0] * gm, fm[0] - fp[0])
    n = KFD * beta ** 1.5 * np.sum(base * diff, axis=1)
    dn = KFD * beta ** 1.5 * np.sum(base * (fm[1] + fp[1]), axis=1)
    return n, dn


# ---------------------------------------------------------------------------
# charge neutrality: eta(d, T)
# ---------------------------------------------------------------------------
def solve_eta(d, T, tol=1e-13, maxit=200):
    """eta with n_- - n_+ = N_A d at each (d, T): Newton on log n_net, in eta
    (beta < BETA_PAIR) or in phi = eta + 1/beta (pair regime), to tol relative
    (the quadrature's own ~1e-15 wobble as the nodes follow eta can leave the
    last steps alternating at a few 1e-15)."""
    d = np.atleast_1d(np.asarray(d, dtype=np.float64))
    T = np.broadcast_to(np.asarray(T, dtype=np.float64), d.shape).copy()
    beta = KERG * T / MEC2
    target = np.log(AVO * d)
    # initial guess: the larger of the non-degenerate and the degenerate (T = 0) estimates
    nq = 2.0 * (2.0 * math.pi * ME * KERG * T / H_PLANCK ** 2) ** 1.5
    eta_nd = np.log(AVO * d / nq)
    xf = H_PLANCK * (3.0 * AVO * d / (8.0 * math.pi)) ** (1.0 / 3.0) / (ME * CLIGHT)
    eta_dg = (np.sqrt(1.0 + xf * xf) - 1.0) / beta
    eta = np.maximum(eta_nd, eta_dg)
    pair = beta >= BETA_PAIR
    phi = np.where(pair, np.maximum(eta + 1.0 / beta, 1e-300), 0.0)
    done = np.zeros(d.shape, dtype=bool)
    for _ in range(maxit):
        e_cur = np.where(pair, phi - 1.0 / beta, eta)
        ph_cur = np.where(pair, phi, e_cur + 1.0 / beta)
        n, dn = _net_density(e_cur, ph_cur, beta)
        with np.errstate(divide="ignore", invalid="ignore"):
            step = (np.log(n) - target) * n / dn
        step = np.where(np.isfinite(step), step, 0.0)
        # phi_new = phi - step: at least phi / 2 in the pair regime (phi > 0), at most 2 phi + 50; eta moves by 50 at most
        step_p = np.clip(step, -(phi + 50.0), 0.5 * phi)
        step_e = np.clip(step, -50.0, 50.0)
        new_phi = np.where(pair & ~done, phi - step_p, phi)
        new_eta = np.where(~pair & ~done, eta - step_e, eta)
        conv = np.where(pair, np.abs(step_p) <= tol * np.maximum(phi, 1e-300) + 1e-300,
                        np.abs(step_e) <= tol * np.maximum(1.0, np.abs(eta)))
        phi, eta = new_phi, new_eta
        done |= conv
        if done.all():
            break
    if not done.all():
        raise RuntimeError(f"eta did not converge at {int((~done).sum())} nodes")
    return np.where(pair, phi - 1.0 / beta, eta), np.where(pair, phi, eta + 1.0 / beta), beta


# ---------------------------------------------------------------------------
# jets: truncated Taylor polynomials in (u, v) = (delta d, delta T)
# ---------------------------------------------------------------------------
_IDX = [(i, j) for s in range(ORDER + 1) for i in range(s, -1, -1) for j in [s - i]]
_POS = {ij: k for k, ij in enumerate(_IDX)}
_MUL = [(_POS[(i1 + i2, j1 + j2)], _POS[(i1, j1)], _POS[(i2, j2)])
        for (i1, j1) in _IDX for (i2, j2) in _IDX if i1 + i2 + j1 + j2 <= ORDER]


class Jet:
    """c[k] is the coefficient of u^i v^j, (i, j) = _IDX[k]; each an array over the nodes."""

    def __init__(self, c):
        self.c = c

    @staticmethod
    def const(a, n):
        c = np.zeros((len(_IDX), n))
        c[0] = a
        return Jet(c)

    def __add__(self, o):
        if isinstance(o, Jet):
            return Jet(self.c + o.c)
        c = self.c.copy()
        c[0] = c[0] + o
        return Jet(c)

    __radd__ = __add__

    def __neg__(self):
        return Jet(-self.c)

    def __sub__(self, o):
        return self + (-o)

    def __rsub__(self, o):
        return (-self) + o

    def __mul__(self, o):
        if not isinstance(o, Jet):
            return Jet(self.c * o)
        c = np.zeros_like(self.c)
        for k, a, b in _MUL:
            c[k] += self.c[a] * o.c[b]
        return Jet(c)

    __rmul__ = __mul__

    def nonconst(self):
        c = self.c.copy()
        c[0] = 0.0
        return Jet(c)

    def deriv(self, i, j):
        """d^(i+j) / du^i dv^j at the expansion point."""
        return self.c[_POS[(i, j)]] * math.factorial(i) * math.factorial(j)


def _jet_fun(x: Jet, derivs):
    """g(x) for a jet x, given g and its derivatives at x's constant term: derivs[m] = g^(m)."""
    dx = x.nonconst()
    out = Jet.const(derivs[0], x.c.shape[1])
    p = None
    for m in range(1, ORDER + 1):
        p = dx if p is None else p * dx
        out = out + p * (derivs[m] / math.factorial(m))
    return out


def _jet_vars(shape):
    """Jets of the two expansion variables themselves."""
    a = Jet(np.zeros((len(_IDX),) + shape))
    a.c[_POS[(1, 0)]] = 1.0
    b = Jet(np.zeros((len(_IDX),) + shape))
    b.c[_POS[(0, 1)]] = 1.0
    return a, b


def _fermi_y(y):
    """f(y) = 1/(exp(y) + 1) and the entropy per state sigma(y) = -f ln f - (1-f) ln(1-f),
    each with its first three y-derivatives (sigma' = -y f (1-f))."""
    e = np.exp(-np.abs(y))
    f = np.where(y > 0, e / (1.0 + e), 1.0 / (1.0 + e))
    g = np.where(y > 0, 1.0 / (1.0 + e), e / (1.0 + e))
    fg = f * g
    l1 = np.log1p(e)
    lnf = np.where(y > 0, -y - l1, -l1)
    lng = np.where(y > 0, -l1, y - l1)
    sig = -f * lnf - g * lng
    fm = f - g
    return ([f, -fg, fg * (g - f), -fg * (1.0 - 6.0 * fg)],
            [sig, -y * fg, -fg * (1.0 + y * fm), -fg * (2.0 * fm + y * fm * fm - 2.0 * y * fg)])


def _species_moments(eta_s, beta0):
    """Jets in (delta psi_s, delta beta) of n, P, E and S = s / k of one species,
    psi_s = eta_s * beta the chemical potential over m_e c^2.

    With eps = beta x the energy over m_e c^2, n = K (M_1/2 + M_3/2),
    P = 2/3 K m_e c^2 (M_3/2 + M_5/2 / 2), E = K m_e c^2 (M_3/2 + M_5/2),
    M_k = int eps^k sqrt(1 + eps/2) f((eps - psi) / beta) d eps, and the
    entropy density s = k K int (eps^1/2 + eps^3/2) sqrt(1 + eps/2) sigma d eps.
    In these variables the temperature enters through the Fermi factor's
    width alone, so thermal derivatives are Fermi-surface integrals and do not
    cancel against the degenerate bulk."""
    x, y, w = _nodes(eta_s)
    r = (1.0 / beta0)[:, None]
    eps = beta0[:, None] * x
    se = np.sqrt(eps)
    wt = beta0[:, None] * w * np.sqrt(1.0 + 0.5 * eps)        # d eps sqrt(1 + eps/2)
    dens = wt * se * (1.0 + eps)
    p32 = wt * eps * se
    p52 = p32 * eps
    # y = (eps - psi) / beta at psi0 + a, beta0 + b: (y0 - a r)(1 - b r + b^2 r^2 - b^3 r^3)
    dy = Jet(np.zeros((len(_IDX),) + x.shape))
    dy.c[_POS[(1, 0)]] = -r
    dy.c[_POS[(0, 1)]] = -y * r
    dy.c[_POS[(1, 1)]] = r * r
    dy.c[_POS[(0, 2)]] = y * r * r
    dy.c[_POS[(1, 2)]] = -r * r * r
    dy.c[_POS[(0, 3)]] = -y * r * r * r
    dy2 = dy * dy
    dy3 = dy2 * dy
    fd, sd = _fermi_y(y)

    def series(dv):
        c = dy.c * dv[1] + dy2.c * (0.5 * dv[2]) + dy3.c * (dv[3] / 6.0)
        c[0] = c[0] + dv[0]
        return c

    fj = series(fd)
    sj = series(sd)
    n = Jet(KFD * np.sum(fj * dens[None], axis=2))
    P = Jet((2.0 / 3.0) * KFD * MEC2 * np.sum(fj * (p32 + 0.5 * p52)[None], axis=2))
    E = Jet(KFD * MEC2 * np.sum(fj * (p32 + p52)[None], axis=2))
    S = Jet(KFD * np.sum(sj * dens[None], axis=2))
    return n, P, E, S


def _compose_ab(Q: Jet, da: Jet, db: Jet):
    """Q(a0 + da, b0 + db) for Q a jet in (a, b) whose coefficients are Taylor coefficients."""
    n = da.c.shape[1]
    pa = [Jet.const(1.0, n)]
    pb = [Jet.const(1.0, n)]
    for _ in range(ORDER):
        pa.append(pa[-1] * da)
        pb.append(pb[-1] * db)
    out = Jet.const(0.0, n)
    for k, (i, j) in enumerate(_IDX):
        out = out + (pa[i] * pb[j]) * Q.c[k]
    return out


CHUNK = 96   # nodes per batch (bounds the per-node jet arrays at a few hundred MB)


def node_values(d, T):
    """The 21 table quantities at nodes (d, T), in the order of the file's four blocks,
    and the jets they come from (for the consistency checks)."""
    d = np.atleast_1d(np.asarray(d, dtype=np.float64))
    T = np.broadcast_to(np.asarray(T, dtype=np.float64), d.shape).copy()
    if d.size > CHUNK:
        parts = [node_values(d[i:i + CHUNK], T[i:i + CHUNK]) for i in range(0, d.size, CHUNK)]
        vals = [[np.concatenate([p[0][b][q] for p in parts]) for q in range(len(parts[0][0][b]))]
                for b in range(len(parts[0][0]))]
        jets = {k: Jet(np.concatenate([p[1][k].c for p in parts], axis=1)) for k in parts[0][1]}
        return vals, jets
    npt = d.size
    eta0, phi0, beta0 = solve_eta(d, T)
    pair = beta0 >= BETA_PAIR
    psi0 = np.where(pair, phi0 * beta0 - 1.0, eta0 * beta0)
    etap0 = -phi0 - 1.0 / beta0                                   # positrons: psi_+ = -psi - 2
    nm_ab, Pm_ab, Em_ab, Sm_ab = _species_moments(eta0, beta0)
    np_ab, Pp_ab, Ep_ab, Sp_ab = _species_moments(etap0, beta0)
    u, v = _jet_vars((npt,))
    d_j = u + d
    T_j = v + T
    dbeta = v * (KERG / MEC2)
    # neutrality n_-(psi) - n_+(-psi - 2) = N_A d, solved for psi's jet order by order
    dn0 = nm_ab.c[_POS[(1, 0)]] + np_ab.c[_POS[(1, 0)]]
    dpsi = Jet(np.zeros((len(_IDX), npt)))
    for _ in range(ORDER):
        r = (_compose_ab(nm_ab, dpsi, dbeta) - _compose_ab(np_ab, -dpsi, dbeta) - AVO * d_j).nonconst()
        dpsi = dpsi - r * (1.0 / dn0)
    P = _compose_ab(Pm_ab, dpsi, dbeta) + _compose_ab(Pp_ab, -dpsi, dbeta)
    Ekin = _compose_ab(Em_ab, dpsi, dbeta) + _compose_ab(Ep_ab, -dpsi, dbeta)
    npos = _compose_ab(np_ab, -dpsi, dbeta)
    xn = _compose_ab(nm_ab, dpsi, dbeta) + npos
    S = _compose_ab(Sm_ab, dpsi, dbeta) + _compose_ab(Sp_ab, -dpsi, dbeta)
    inv_d = _jet_fun(d_j, [1.0 / d, -1.0 / d ** 2, 2.0 / d ** 3, -6.0 / d ** 4])
    beta_j = dbeta + beta0
    inv_b = _jet_fun(beta_j, [1.0 / beta0, -1.0 / beta0 ** 2, 2.0 / beta0 ** 3, -6.0 / beta0 ** 4])
    psi_j = dpsi + psi0
    eta_j = psi_j * inv_b
    eta_j.c[0] = eta0                                             # as solved (psi0 / beta0 rounds)
    s = KERG * S * inv_d
    p0 = P.deriv(0, 0)
    pd, pt = P.deriv(1, 0), P.deriv(0, 1)
    pdd, pdt, ptt = P.deriv(2, 0), P.deriv(1, 1), P.deriv(0, 2)
    pddt, pdtt = P.deriv(2, 1), P.deriv(1, 2)
    d2, d3 = d * d, d * d * d
    f = AVO * MEC2 * psi0 - p0 / d
    vals = [
        [f, p0 / d2, -s.deriv(0, 0), pd / d2 - 2.0 * p0 / d3, -s.deriv(0, 1), pt / d2,
         pdt / d2 - 2.0 * pt / d3, ptt / d2, pdtt / d2 - 2.0 * ptt / d3],
        [pd, pdd, pdt, pddt],
        [eta0, eta_j.deriv(1, 0), eta_j.deriv(0, 1), eta_j.deriv(1, 1)],
        [xn.deriv(0, 0), xn.deriv(1, 0), xn.deriv(0, 1), xn.deriv(1, 1)],
    ]
    return vals, {"s_jet": s, "P_jet": P, "psi_jet": psi_j, "eta_jet": eta_j, "E_jet": Ekin, "npos_jet": npos}


def fd_tables(rows=None, cols=None, workers=None):
    """The 21 tables as (JMAX, IMAX) arrays in read order.  With ``rows`` /
    ``cols`` (temperature / density indices) only that window is computed and
    the other nodes keep the analytic non-degenerate values of ``helm_table``
    (a window around the states a short run visits, for tests)."""
    d1, t1 = _ht.grid()
    rows = list(range(JMAX)) if rows is None else list(rows)
    cols = np.arange(IMAX) if cols is None else np.asarray(list(cols))
    out = [[np.array(a) for a in block] for block in _ht.ideal_nd_tables()]
    args = [(t1[j], d1[cols]) for j in rows]
    if workers and workers > 1 and len(rows) > 1:
        import importlib.machinery
        import multiprocessing as mp
        import sys

        # spawn workers import _row by its module name: run as a script (ensure_table
        # does) when this module was loaded from a file path under a name a fresh
        # interpreter cannot import
        top = __name__.split(".")[0]
        if __name__ != "__main__" and importlib.machinery.PathFinder.find_spec(top, sys.path) is None:
            raise RuntimeError("helm_fd: a worker pool needs the module importable by name; "
                               "use ensure_table() or run helm_fd.py as a script")

        with mp.get_context("spawn").Pool(workers) as pool:
            res = pool.map(_row, args)
    else:
        res = [_row(a) for a in args]
    for j, blocks in zip(rows, res):
        for b, block in enumerate(blocks):
            for q, arr in enumerate(block):
                out[b][q][j, cols] = arr
    return out


def _row(args):
    t, d = args
    vals, _ = node_values(d, np.full_like(d, t))
    return vals


def write_table(path: str = DEFAULT_PATH, workers: int | None = None, rows=None, cols=None) -> str:
    """Write the Fermi-Dirac table (or a window of it, see fd_tables) to ``path``
    atomically and return the path."""
    if workers is None:
        workers = max(1, min(16, os.cpu_count() or 1))
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tabs = fd_tables(rows=rows, cols=cols, workers=workers)
    tmp = f"{path}.tmp.{os.getpid()}"
    with open(tmp, "w") as fp:
        for block in tabs:
            cols_ = np.stack([b.reshape(-1) for b in block], axis=1)  # rows: j slow, i fast
            np.savetxt(fp, cols_, fmt="%.17e")
    os.replace(tmp, path)
    return path


def ensure_table(path: str = DEFAULT_PATH) -> str:
    """The table at ``path``, generated first when it is missing.  The generation
    runs this file as a script in a process of its own: its worker pool is
    started with ``spawn``, whose workers must import the row function by name,
    and the package directory (``mini-castro_b200``) is not importable by name."""
    if not os.path.exists(path):
        import subprocess
        import sys

        subprocess.run([sys.executable, os.path.abspath(__file__), path], check=True, stdout=subprocess.DEVNULL)
    return path


if __name__ == "__main__":
    import sys

    p = write_table(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_PATH)
    print(p, _ht.sha256(p))
