"""Exact solution of the Riemann problem of an ideal gas (test infrastructure).

The standard construction (Toro, "Riemann Solvers and Numerical Methods for
Fluid Dynamics", ch. 4): the star pressure p* is the root of
f_L(p) + f_R(p) + (u_R - u_L) = 0, with f_K the shock (Rankine-Hugoniot) or
rarefaction (isentropic) branch of side K, solved here by bisection on a
bracketing interval; the solution at x/t is sampled from the wave pattern.
Written for the known-answer tests of the hydro scheme; not used by the
library.
"""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho, pk, ck, g):
    if p > pk:      # shock
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        return (p - pk) * math.sqrt(A / (p + B))
    return 2.0 * ck / (g - 1.0) * ((p / pk) ** ((g - 1.0) / (2.0 * g)) - 1.0)   # rarefaction


def star_state(left, right, g):
    """(p*, u*) of the Riemann problem between left = (rho, u, p) and right."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def F(p):
        return _f(p, rl, pl, cl, g) + _f(p, rr, pr, cr, g) + (ur - ul)

    lo, hi = 1e-12 * min(pl, pr), 10.0 * max(pl, pr)
    assert F(lo) < 0.0 < F(hi), "no vacuum-free star state in the bracket"
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if F(mid) > 0.0:
            hi = mid
        else:
            lo = mid
    p = 0.5 * (lo + hi)
    u = 0.5 * (ul + ur) + 0.5 * (_f(p, rr, pr, cr, g) - _f(p, rl, pl, cl, g))
    return p, u


def sample(left, right, g, s):
    """(rho, u, p) at the similarity coordinates s = (x - x0) / t (array)."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    ps, us = star_state(left, right, g)
    gm = (g - 1.0) / (g + 1.0)
    out = np.zeros((len(s), 3))
    for n, x in enumerate(np.asarray(s, dtype=float)):
        if x <= us:      # left of the contact
            if ps > pl:  # left shock
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                if x <= sl:
                    out[n] = (rl, ul, pl)
                else:
                    out[n] = (rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps)
            else:        # left rarefaction
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                if x <= ul - cl:
                    out[n] = (rl, ul, pl)
                elif x >= us - csl:
                    out[n] = (rl * (ps / pl) ** (1.0 / g), us, ps)
                else:    # inside the fan
                    c = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * (ul - x))
                    u = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * ul + x)
                    r = rl * (c / cl) ** (2.0 / (g - 1.0))
                    out[n] = (r, u, pl * (c / cl) ** (2.0 * g / (g - 1.0)))
        else:            # right of the contact
            if ps > pr:  # right shock
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                if x >= sr:
                    out[n] = (rr, ur, pr)
                else:
                    out[n] = (rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps)
            else:        # right rarefaction
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                if x >= ur + cr:
                    out[n] = (rr, ur, pr)
                elif x <= us + csr:
                    out[n] = (rr * (ps / pr) ** (1.0 / g), us, ps)
                else:
                    c = 2.0 / (g + 1.0) * (cr - 0.5 * (g - 1.0) * (ur - x))
                    u = 2.0 / (g + 1.0) * (-cr + 0.5 * (g - 1.0) * ur + x)
                    r = rr * (c / cr) ** (2.0 / (g - 1.0))
                    out[n] = (r, u, pr * (c / cr) ** (2.0 * g / (g - 1.0)))
    return out
