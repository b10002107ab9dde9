"""Reverse mode on the GPU.

* Each <routine>_adj entry point against central finite differences of its
  forward entry point (same inputs, seeded output weights w and input
  direction v: <J^T w, v> vs (w.f(x+hv) - w.f(x-hv)) / 2h), on the states of a
  developed 16^3 Sedov blast.
* The whole-run gradient (castro_adj_*) of the shell kinetic energy with
  respect to the blast energy, the ambient density and the per-zone density
  perturbation, against central finite differences (relative step 1e-6) of the
  GPU forward along seeded directions, and against finite differences of the
  oracle's forward.
* The torch.autograd.Function wrapper.

Finite differences of a shock-capturing scheme are spoiled wherever a limiter
or Riemann branch switches inside the difference stencil; the per-routine
checks therefore take the best of three step sizes (h, 10h, h/10): a correct
adjoint matches one of them to ~1e-7, a wrong one matches none.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_harness import from_dev, sborder_from_domain, to_dev

pytestmark = pytest.mark.gpu

NS = 2
NV, QV, NQAUX, NGDNV = 7 + NS, 8 + NS, 4, 6
QGAME, QTEMP, UTEMP = 4, 7, 6
N = 16
BX = ((0, 0, 0), (N - 1, N - 1, N - 1))


def grow(b, g):
    return (tuple(x - g for x in b[0]), tuple(x + g for x in b[1]))


def ebx(d):
    hi = list(BX[1])
    hi[d] += 1
    return (BX[0], tuple(hi))


def growv(b, v):
    return (tuple(x - g for x, g in zip(b[0], v)), tuple(x + g for x, g in zip(b[1], v)))


TBX = {}
for a, grows in ((0, ((0, 1, 1), (0, 0, 1), (0, 1, 0))), (1, ((0, 0, 1), (1, 0, 1), (1, 0, 0))),
                 (2, ((0, 1, 0), (1, 0, 0), (1, 1, 0)))):
    for b in range(3):
        TBX[(a, b)] = growv(ebx(a), grows[b])
QBX, OBX = grow(BX, 4), grow(BX, 1)


def shape(b, nc):
    return (nc,) + tuple(h - l + 1 for l, h in reversed(list(zip(*b))))


def zeros(b, nc):
    import torch

    return torch.zeros(shape(b, nc), dtype=torch.float64, device="cuda")


@pytest.fixture(scope="module")
def env(pkg, table):
    """A developed 16^3 outflow Sedov state: cleaned Sborder, q, qaux, traces, fluxes."""
    import torch

    K = pkg.castro
    L = K.init(*pkg.configs.NET2, table)
    cfg = pkg.configs.sedov64(scale=4)
    sim = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    sim.init_data()
    sim.step(6)
    inst = cfg["instances"][0]
    G = K.assemble(inst, sim.box_states()[0])
    sim.close()
    # seeded noise everywhere: the ambient of the blast is exactly uniform at rest, where
    # every limiter sits on a tie (equal neighbours, zero slopes) that a finite
    # difference would break but an adjoint cannot see
    rng = np.random.default_rng(3)
    r = lambda: rng.standard_normal(G.shape[:3])
    G[..., 0] *= 1 + 1e-3 * r()
    mscale = np.abs(G[..., 1:4]).max()
    for c in (1, 2, 3):
        G[..., c] += 1e-3 * mscale * r()
    G[..., 5] *= 1 + 1e-3 * r()
    G[..., 4] = G[..., 5] + 0.5 * (G[..., 1] ** 2 + G[..., 2] ** 2 + G[..., 3] ** 2) / G[..., 0]
    for c in range(7, 7 + NS):
        G[..., c] *= 1 + 1e-3 * r()
    sb = to_dev(sborder_from_domain(G, inst["dom_lo"], BX[0], BX[1], inst["bc"]))
    for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
        K.call(L, name, QBX[0], QBX[1], sb, QBX[0], QBX[1])
    q, qa = zeros(QBX, QV), zeros(QBX, NQAUX)
    K.call(L, "ctoprim", QBX[0], QBX[1], sb, QBX[0], QBX[1], q, QBX[0], QBX[1], qa, QBX[0], QBX[1])
    # gamma_1 is 4/3 to the last bit wherever radiation dominates: break those ties too
    # (the routines under test take qaux as an independent input)
    gq = torch.Generator(device="cuda").manual_seed(4)
    for c in (0, 1):
        qa[c] *= 1 + 1e-3 * torch.randn(qa[c].shape, dtype=torch.float64, device="cuda", generator=gq)
    dx = [1.0 / N] * 3
    dt = 0.4 * sim_dt_guess(L, K, sb, dx)
    qm = {d: zeros(OBX, QV) for d in range(3)}
    qp = {d: zeros(OBX, QV) for d in range(3)}
    for d in range(3):
        K.call(L, "trace_ppm", OBX[0], OBX[1], BX[0], BX[1], d + 1, q, QBX[0], QBX[1], qa, QBX[0], QBX[1], qm[d],
               OBX[0], OBX[1], qp[d], OBX[0], OBX[1], BX[0], BX[1], dx, float(dt))
    torch.cuda.synchronize()
    return dict(L=L, K=K, sb=sb, q=q, qa=qa, qm=qm, qp=qp, dx=dx, dt=float(dt), table=table)


def sim_dt_guess(L, K, sb, dx):
    import torch

    d = torch.full((1,), 1e300, dtype=torch.float64, device="cuda")
    K.call(L, "estdt", BX[0], BX[1], sb, QBX[0], QBX[1], dx, d)
    return float(d.item()) * 0.5


def fd_best(f, x, v, h, ad):
    vals = []
    for hh in (h, 10 * h, 0.1 * h):
        vals.append((f(x, v, hh) - f(x, v, -hh)) / (2 * hh))
    return min(vals, key=lambda t: abs(t - ad))


def check_routine(fwd, adj, inputs, out_shapes, masks=None, seed=0, h=1e-6, tol=1e-5, scalars=(), probes=6):
    """fwd(inputs) -> dict of outputs; adj(inputs, wbar) -> dict of input adjoints
    (tensors, or floats for the names in `scalars`).

    Single-entry probes: for `probes` seeded entries of each input (those the
    adjoint reports as nonzero, so the probe exercises a real dependence) the
    adjoint entry is compared with the central difference of w.f along that
    entry alone; a probe perturbs only the branches inside its own stencil.
    At least 90% of the probes must agree to `tol` and every probe to 1e-2."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    w = {k: torch.randn(s, dtype=torch.float64, device="cuda", generator=g) for k, s in out_shapes.items()}
    for k, comps in (masks or {}).items():
        for c in comps:
            w[k][c] = 0.0
    xb = adj(inputs, w)
    rng = np.random.default_rng(seed)
    # outputs span many decades (ambient 1e13 .. blast 1e52 erg/cm^3): difference
    # against the unperturbed outputs so a local change is not lost in the sum
    y0 = fwd(dict(inputs))

    def f(x, vv, hh):
        xi = dict(x)
        k, idx, step = vv
        if k in scalars:
            xi[k] = x[k] + hh * step
        else:
            t = x[k].clone()
            t.view(-1)[idx] += hh * step
            xi[k] = t
        y = fwd(xi)
        return sum(float((w[kk] * (y[kk] - y0[kk])).sum()) for kk in w)

    errs, bad = [], []
    for k in inputs:
        if k in scalars:
            sel = [None]
        else:
            if k not in xb:
                continue
            # entries whose first-order contribution |xb * x| is resolvable by a
            # central difference: at least 1e-6 of the largest one of this input
            contrib = (xb[k] * inputs[k].abs().clamp_min(1e-300)).abs().view(-1)
            cmax = float(contrib.max())
            if cmax == 0.0:
                continue
            nz = torch.nonzero(contrib >= 1e-6 * cmax).view(-1).cpu().numpy()
            sel = rng.choice(nz, size=min(probes, len(nz)), replace=False)
        for idx in sel:
            if k in scalars:
                step = abs(inputs[k]) or 1.0
                ad = xb.get(k, 0.0) * step
            else:
                xv = float(inputs[k].view(-1)[int(idx)])
                step = abs(xv) if xv != 0.0 else 1.0
                ad = float(xb[k].view(-1)[int(idx)]) * step
            fdv = fd_best(f, inputs, (k, None if idx is None else int(idx), step), h, ad)
            floor = 1e-9 * (abs(ad) if k in scalars else cmax)
            e = abs(ad - fdv) / max(abs(ad), abs(fdv), floor, 1e-300)
            errs.append(e)
            if e > tol:
                where = "" if k in scalars else "comp %d zone %s" % (
                    int(idx) // int(np.prod(inputs[k].shape[1:])),
                    np.unravel_index(int(idx) % int(np.prod(inputs[k].shape[1:])), inputs[k].shape[1:])[::-1])
                bad.append(f"{k} {where}: ad {ad:.6e} fd {fdv:.6e}")
    errs = np.array(errs)
    assert len(errs) > 0
    frac_ok = float((errs <= tol).mean())
    assert frac_ok >= 0.9 and errs.max() <= 1e-2, \
        f"probe errors {np.sort(errs)[-5:]} ({frac_ok:.0%} within {tol:g}); " + "; ".join(bad)
    return errs


# ---------------------------------------------------------------------------
# per-routine adjoints
# ---------------------------------------------------------------------------
def test_ctoprim_adj(env):
    K, L = env["K"], env["L"]

    def fwd(x):
        q, qa = zeros(QBX, QV), zeros(QBX, NQAUX)
        K.call(L, "ctoprim", QBX[0], QBX[1], x["u"], QBX[0], QBX[1], q, QBX[0], QBX[1], qa, QBX[0], QBX[1])
        return {"q": q, "qa": qa}

    def adj(x, w):
        ub = zeros(QBX, NV)
        K.call(L, "ctoprim_adj", QBX[0], QBX[1], x["u"], QBX[0], QBX[1], w["q"], QBX[0], QBX[1], w["qa"], QBX[0],
               QBX[1], ub, QBX[0], QBX[1])
        ub[UTEMP] = 0.0
        return {"u": ub}

    u = env["sb"].clone()
    check_routine(lambda x: fwd({"u": _no_temp(x["u"], u)}), adj, {"u": u}, {"q": shape(QBX, QV), "qa": shape(QBX, NQAUX)})


def _no_temp(x, base):
    """Keep the Newton guess channel fixed: UTEMP is not a differentiable input."""
    y = x.clone()
    y[UTEMP] = base[UTEMP]
    return y


def test_clean_state_adj(env):
    K, L = env["K"], env["L"]
    u0 = env["sb"].clone()

    def fwd(x):
        u = _no_temp(x["u"], u0)
        for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
            K.call(L, name, QBX[0], QBX[1], u, QBX[0], QBX[1])
        return {"u": u}

    def adj(x, w):
        ub = w["u"].clone()
        K.call(L, "clean_state_adj", QBX[0], QBX[1], x["u"], QBX[0], QBX[1], ub, QBX[0], QBX[1])
        ub[UTEMP] = 0.0
        return {"u": ub}

    check_routine(fwd, adj, {"u": u0}, {"u": shape(QBX, NV)}, masks={"u": [UTEMP]}, h=1e-6)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_trace_ppm_adj(env, d):
    K, L, dx = env["K"], env["L"], env["dx"]

    def fwd(x):
        qm, qp = zeros(OBX, QV), zeros(OBX, QV)
        K.call(L, "trace_ppm", OBX[0], OBX[1], BX[0], BX[1], d + 1, x["q"], QBX[0], QBX[1], x["qa"], QBX[0], QBX[1],
               qm, OBX[0], OBX[1], qp, OBX[0], OBX[1], BX[0], BX[1], dx, float(x["dt"]))
        return {"qm": qm, "qp": qp}

    def adj(x, w):
        import torch

        qb, qab = zeros(QBX, QV), zeros(QBX, NQAUX)
        dtb = torch.zeros(1, dtype=torch.float64, device="cuda")
        K.call(L, "trace_ppm_adj", OBX[0], OBX[1], BX[0], BX[1], d + 1, x["q"], QBX[0], QBX[1], x["qa"], QBX[0],
               QBX[1], w["qm"], OBX[0], OBX[1], w["qp"], OBX[0], OBX[1], qb, QBX[0], QBX[1], qab, QBX[0], QBX[1], dx,
               float(x["dt"]), dtb)
        return {"q": qb, "qa": qab, "dt": float(dtb.item())}

    check_routine(fwd, adj, {"q": env["q"], "qa": env["qa"], "dt": env["dt"]},
                  {"qm": shape(OBX, QV), "qp": shape(OBX, QV)}, masks={"qm": [QGAME, QTEMP], "qp": [QGAME, QTEMP]},
                  scalars=("dt",), seed=d, probes=12)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_compute_flux_adj(env, d):
    K, L = env["K"], env["L"]
    b = TBX[(d, d)]

    def fwd(x):
        fx, qi, qg = zeros(OBX, NV), zeros(OBX, QV), zeros(OBX, NGDNV)
        K.call(L, "compute_flux", b[0], b[1], x["ql"], OBX[0], OBX[1], x["qr"], OBX[0], OBX[1], fx, OBX[0], OBX[1],
               qi, OBX[0], OBX[1], qg, OBX[0], OBX[1], x["qa"], QBX[0], QBX[1], d + 1)
        return {"f": fx, "g": qg}

    def adj(x, w):
        qlb, qrb, qab = zeros(OBX, QV), zeros(OBX, QV), zeros(QBX, NQAUX)
        K.call(L, "compute_flux_adj", b[0], b[1], x["ql"], OBX[0], OBX[1], x["qr"], OBX[0], OBX[1], x["qa"], QBX[0],
               QBX[1], w["f"], OBX[0], OBX[1], w["g"], OBX[0], OBX[1], qlb, OBX[0], OBX[1], qrb, OBX[0], OBX[1], qab,
               QBX[0], QBX[1], d + 1)
        return {"ql": qlb, "qr": qrb, "qa": qab}

    check_routine(fwd, adj, {"ql": env["qm"][d], "qr": env["qp"][d], "qa": env["qa"]},
                  {"f": shape(OBX, NV), "g": shape(OBX, NGDNV)}, masks={"f": [UTEMP]}, seed=10 + d)


@pytest.mark.parametrize("d", [0, 2])
def test_compute_flux_adj_momentum_pressure(env, d):
    """The same probe with the interface pressure in the normal momentum flux
    (castro_set_momentum_flux_pressure; the reference has none)."""
    L = env["L"]
    L.castro_set_momentum_flux_pressure(1)
    try:
        test_compute_flux_adj(env, d)
    finally:
        L.castro_set_momentum_flux_pressure(0)


def _riemann1(env, d):
    K, L = env["K"], env["L"]
    b = TBX[(d, d)]
    fx, qi, qg = zeros(OBX, NV), zeros(OBX, QV), zeros(OBX, NGDNV)
    K.call(L, "compute_flux", b[0], b[1], env["qm"][d], OBX[0], OBX[1], env["qp"][d], OBX[0], OBX[1], fx, OBX[0],
           OBX[1], qi, OBX[0], OBX[1], qg, OBX[0], OBX[1], env["qa"], QBX[0], QBX[1], d + 1)
    return fx, qg


@pytest.mark.parametrize("pair", [(0, 1), (2, 0), (1, 2)])
def test_trans1_adj(env, pair):
    import torch

    K, L = env["K"], env["L"]
    d, t = pair            # flux direction d corrects the states normal to t
    b = TBX[(t, d)]
    f1, g1 = _riemann1(env, d)
    cdtdx = env["dt"] / env["dx"][d] / 3.0

    def fwd(x):
        qmo, qpo = zeros(OBX, QV), zeros(OBX, QV)
        K.call(L, "trans1", b[0], b[1], d + 1, t + 1, x["qm"], OBX[0], OBX[1], qmo, OBX[0], OBX[1], x["qp"], OBX[0],
               OBX[1], qpo, OBX[0], OBX[1], x["qa"], QBX[0], QBX[1], x["f"], OBX[0], OBX[1], x["g"], OBX[0], OBX[1],
               float(x["c"]))
        return {"qmo": qmo, "qpo": qpo}

    def adj(x, w):
        qmb, qpb, qab, fb, gb = zeros(OBX, QV), zeros(OBX, QV), zeros(QBX, NQAUX), zeros(OBX, NV), zeros(OBX, NGDNV)
        cb = torch.zeros(1, dtype=torch.float64, device="cuda")
        K.call(L, "trans1_adj", b[0], b[1], d + 1, t + 1, x["qm"], OBX[0], OBX[1], x["qp"], OBX[0], OBX[1], x["qa"],
               QBX[0], QBX[1], x["f"], OBX[0], OBX[1], x["g"], OBX[0], OBX[1], float(x["c"]), w["qmo"], OBX[0], OBX[1],
               w["qpo"], OBX[0], OBX[1], qmb, OBX[0], OBX[1], qpb, OBX[0], OBX[1], qab, QBX[0], QBX[1], fb, OBX[0],
               OBX[1], gb, OBX[0], OBX[1], cb)
        return {"qm": qmb, "qp": qpb, "qa": qab, "f": fb, "g": gb, "c": float(cb.item())}

    check_routine(fwd, adj, {"qm": env["qm"][t], "qp": env["qp"][t], "qa": env["qa"], "f": f1, "g": g1, "c": cdtdx},
                  {"qmo": shape(OBX, QV), "qpo": shape(OBX, QV)}, masks={"qmo": [QGAME, QTEMP], "qpo": [QGAME, QTEMP]},
                  scalars=("c",), seed=20 + d)


def test_trans2_adj(env):
    import torch

    K, L = env["K"], env["L"]
    d, t1, t2 = 0, 1, 2
    # transverse-corrected fluxes of directions t1 | t2 and t2 | t1 stand in for the riemann2 outputs
    f2, g2 = _riemann1(env, t1)
    f3, g3 = _riemann1(env, t2)
    c2 = 0.5 * env["dt"] / env["dx"][t1]
    c3 = 0.5 * env["dt"] / env["dx"][t2]
    e = ebx(d)

    def fwd(x):
        qmo, qpo = zeros(OBX, QV), zeros(OBX, QV)
        K.call(L, "trans2", e[0], e[1], d + 1, t1 + 1, t2 + 1, x["qm"], OBX[0], OBX[1], qmo, OBX[0], OBX[1], x["qp"],
               OBX[0], OBX[1], qpo, OBX[0], OBX[1], x["qa"], QBX[0], QBX[1], x["f2"], OBX[0], OBX[1], x["f3"], OBX[0],
               OBX[1], x["g2"], OBX[0], OBX[1], x["g3"], OBX[0], OBX[1], 0.0, float(x["c2"]), float(x["c3"]))
        return {"qmo": qmo, "qpo": qpo}

    def adj(x, w):
        qmb, qpb, qab = zeros(OBX, QV), zeros(OBX, QV), zeros(QBX, NQAUX)
        f2b, f3b, g2b, g3b = zeros(OBX, NV), zeros(OBX, NV), zeros(OBX, NGDNV), zeros(OBX, NGDNV)
        cb = torch.zeros(2, dtype=torch.float64, device="cuda")
        K.call(L, "trans2_adj", e[0], e[1], d + 1, t1 + 1, t2 + 1, x["qm"], OBX[0], OBX[1], x["qp"], OBX[0], OBX[1],
               x["qa"], QBX[0], QBX[1], x["f2"], OBX[0], OBX[1], x["f3"], OBX[0], OBX[1], x["g2"], OBX[0], OBX[1],
               x["g3"], OBX[0], OBX[1], float(x["c2"]), float(x["c3"]), w["qmo"], OBX[0], OBX[1], w["qpo"], OBX[0],
               OBX[1], qmb, OBX[0], OBX[1], qpb, OBX[0], OBX[1], qab, QBX[0], QBX[1], f2b, OBX[0], OBX[1], f3b,
               OBX[0], OBX[1], g2b, OBX[0], OBX[1], g3b, OBX[0], OBX[1], C.c_void_p(cb.data_ptr()),
               C.c_void_p(cb.data_ptr() + 8))
        return {"qm": qmb, "qp": qpb, "qa": qab, "f2": f2b, "f3": f3b, "g2": g2b, "g3": g3b,
                "c2": float(cb[0].item()), "c3": float(cb[1].item())}

    check_routine(fwd, adj, {"qm": env["qm"][d], "qp": env["qp"][d], "qa": env["qa"], "f2": f2, "f3": f3, "g2": g2,
                             "g3": g3, "c2": c2, "c3": c3},
                  {"qmo": shape(OBX, QV), "qpo": shape(OBX, QV)}, masks={"qmo": [QGAME, QTEMP], "qpo": [QGAME, QTEMP]},
                  scalars=("c2", "c3"), seed=30)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_apply_av_and_normalize_adj(env, d):
    K, L, dx = env["K"], env["L"], env["dx"]
    e = ebx(d)
    ge = grow(e, 1)
    f1, _ = _riemann1(env, d)
    # a flux FAB on gebx holding the riemann1 fluxes of the same faces (both FABs start at lo-1)
    fl = zeros(ge, NV)
    fl[:, :f1.shape[1], :f1.shape[2], :f1.shape[3]] = f1
    div = zeros(OBX, 1)
    K.call(L, "divu", OBX[0], OBX[1], env["q"], QBX[0], QBX[1], dx, div, OBX[0], OBX[1])

    def fwd(x):
        f = x["f"].clone()
        K.call(L, "apply_av", e[0], e[1], d + 1, dx, x["div"], OBX[0], OBX[1], x["sb"], QBX[0], QBX[1], f, ge[0], ge[1])
        K.call(L, "normalize_species_fluxes", e[0], e[1], f, ge[0], ge[1])
        return {"f": f}

    def adj(x, w):
        f = x["f"].clone()
        K.call(L, "apply_av", e[0], e[1], d + 1, dx, x["div"], OBX[0], OBX[1], x["sb"], QBX[0], QBX[1], f, ge[0], ge[1])
        fb = w["f"].clone()
        K.call(L, "normalize_species_fluxes_adj", e[0], e[1], f, ge[0], ge[1], fb, ge[0], ge[1])
        divb, sbb = zeros(OBX, 1), zeros(QBX, NV)
        K.call(L, "apply_av_adj", e[0], e[1], d + 1, dx, x["div"], OBX[0], OBX[1], x["sb"], QBX[0], QBX[1], fb, ge[0],
               ge[1], divb, OBX[0], OBX[1], sbb, QBX[0], QBX[1])
        return {"f": fb, "div": divb, "sb": sbb}

    check_routine(fwd, adj, {"f": fl, "div": div, "sb": env["sb"]}, {"f": shape(ge, NV)}, masks={"f": [UTEMP]},
                  seed=40 + d)


def test_fill_hydro_source_and_divu_adj(env):
    K, L, dx = env["K"], env["L"], env["dx"]
    ge = [grow(ebx(d), 1) for d in range(3)]
    import torch

    g = torch.Generator(device="cuda").manual_seed(5)
    fl = [torch.randn(shape(ge[d], NV), dtype=torch.float64, device="cuda", generator=g) for d in range(3)]
    qe = [torch.randn(shape(ge[d], NGDNV), dtype=torch.float64, device="cuda", generator=g) for d in range(3)]
    area = [torch.full(shape(ge[d], 1), dx[1] * dx[2], dtype=torch.float64, device="cuda") for d in range(3)]
    vol = torch.full(shape(BX, 1), dx[0] * dx[1] * dx[2], dtype=torch.float64, device="cuda")

    def fwd(x):
        src = zeros(BX, NV)
        args = []
        for d in range(3):
            args += [x[f"f{d}"], ge[d][0], ge[d][1]]
        for d in range(3):
            args += [x[f"e{d}"], ge[d][0], ge[d][1]]
        for d in range(3):
            args += [area[d], ge[d][0], ge[d][1]]
        K.call(L, "fill_hydro_source", BX[0], BX[1], env["sb"], QBX[0], QBX[1], env["q"], QBX[0], QBX[1], src, BX[0],
               BX[1], *args, vol, BX[0], BX[1], dx, 0.0)
        div = zeros(OBX, 1)
        K.call(L, "divu", OBX[0], OBX[1], x["q"], QBX[0], QBX[1], dx, div, OBX[0], OBX[1])
        return {"src": src, "div": div}

    def adj(x, w):
        fb = [zeros(ge[d], NV) for d in range(3)]
        eb = [zeros(ge[d], NGDNV) for d in range(3)]
        args = []
        for d in range(3):
            args += [x[f"e{d}"], ge[d][0], ge[d][1]]
        for d in range(3):
            args += [area[d], ge[d][0], ge[d][1]]
        outs = []
        for d in range(3):
            outs += [fb[d], ge[d][0], ge[d][1]]
        for d in range(3):
            outs += [eb[d], ge[d][0], ge[d][1]]
        K.call(L, "fill_hydro_source_adj", BX[0], BX[1], w["src"], BX[0], BX[1], *args, vol, BX[0], BX[1], dx, *outs)
        qb = zeros(QBX, QV)
        K.call(L, "divu_adj", OBX[0], OBX[1], dx, w["div"], OBX[0], OBX[1], qb, QBX[0], QBX[1])
        r = {f"f{d}": fb[d] for d in range(3)}
        r.update({f"e{d}": eb[d] for d in range(3)})
        r["q"] = qb
        return r

    x = {f"f{d}": fl[d] for d in range(3)}
    x.update({f"e{d}": qe[d] for d in range(3)})
    x["q"] = env["q"]
    check_routine(fwd, adj, x, {"src": shape(BX, NV), "div": shape(OBX, 1)}, seed=50)


# ---------------------------------------------------------------------------
# whole-run gradients
# ---------------------------------------------------------------------------
def shell_energy_np(G, inst, r0=0.3, r1=0.4):
    n = G.shape[0]
    lo, hi = np.array(inst["problo"]), np.array(inst["probhi"])
    dxs = (hi - lo) / n
    c = 0.5 * (lo + hi)
    ax = [lo[d] + (np.arange(n) + 0.5) * dxs[d] - c[d] for d in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    L = hi[0] - lo[0]
    m = (r >= r0 * L) & (r <= r1 * L)
    ke = 0.5 * (G[..., 1] ** 2 + G[..., 2] ** 2 + G[..., 3] ** 2) / G[..., 0]
    return float((ke * m).sum() * np.prod(dxs))


def _runner(pkg, table, scale, steps, ckpt, exact=False):
    K = pkg.castro
    L = K.init(*pkg.configs.NET2, table, exact=exact)
    cfg = pkg.configs.adjoint64(scale=scale, steps=steps)
    inst = cfg["instances"][0]
    return pkg.adjoint.SedovAdjoint(L, inst, steps, ckpt), inst


def _directions(n, k, seed):
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal(), rng.standard_normal(), rng.standard_normal((n, n, n))) for _ in range(k)]


def test_adjoint_forward_matches_oracle(pkg, table, oracle):
    """The adjoint's own forward is the reference sequence: bit-identical final
    state and dt sequence with the oracle in the exact build."""
    import torch

    run, inst = _runner(pkg, table, 4, 4, 2, exact=True)
    J = run.forward(inst["problem"]["exp_energy"], inst["problem"]["dens_ambient"])
    V = run.final_state().cpu().numpy().transpose(3, 2, 1, 0)
    cfg = pkg.configs.adjoint64(scale=4, steps=4)
    oracle.network_init(*cfg["network"])
    oracle.eos_init(table)
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    dts = [lev.coarse_step(-1.0) for _ in range(4)]
    Go = oracle.assemble(lev, inst)
    np.testing.assert_array_equal(V, Go)
    assert run.dts() == dts
    assert J == pytest.approx(shell_energy_np(Go, inst), rel=1e-13)
    run.close()
    torch.cuda.synchronize()


@pytest.mark.parametrize("scale,steps,ckpt,ndir", [(2, 10, 3, 8)], ids=["32cube_10steps"])
def test_gradient_matches_fd_of_gpu_forward(pkg, table, scale, steps, ckpt, ndir):
    import torch

    run, inst = _runner(pkg, table, scale, steps, ckpt)
    p = inst["problem"]
    E0, R0 = p["exp_energy"], p["dens_ambient"]
    pert0 = run.pert.clone()
    J0 = run.forward(E0, R0, pert0)
    dE, dR, dP = run.backward()
    assert np.isfinite(dE) and np.isfinite(dR) and bool(torch.isfinite(dP).all())
    n = run.n[0]
    h = 1e-6
    errs = []
    for a, b, c in _directions(n, ndir, 11):
        ct = torch.from_numpy(np.ascontiguousarray(c.transpose(2, 1, 0))).cuda()
        ad = dE * E0 * a + dR * R0 * b + float((dP * ct).sum())
        Jp = run.forward(E0 * (1 + h * a), R0 * (1 + h * b), pert0 + h * ct)
        Jm = run.forward(E0 * (1 - h * a), R0 * (1 - h * b), pert0 - h * ct)
        fd = (Jp - Jm) / (2 * h)
        errs.append(abs(ad - fd) / max(abs(ad), abs(fd)))
    print("J", J0, "directional rel errors", ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5, errs
    run.close()


def test_gradient_matches_fd_of_oracle(pkg, table, oracle):
    """dJ along seeded directions from the GPU adjoint vs central finite
    differences of the oracle's forward (16^3, 5 steps)."""
    import torch

    run, inst = _runner(pkg, table, 4, 5, 2)
    p = inst["problem"]
    E0, R0 = p["exp_energy"], p["dens_ambient"]
    run.forward(E0, R0)
    dE, dR, dP = run.backward()
    cfg = pkg.configs.adjoint64(scale=4, steps=5)
    oracle.network_init(*cfg["network"])
    oracle.eos_init(table)
    n = run.n[0]

    def J_oracle(E, R, pert):
        i2 = dict(inst)
        pr = dict(p)
        pr.update(exp_energy=E, dens_ambient=R, pert=np.asfortranarray(pert))
        i2["problem"] = pr
        lev, _ = oracle.level_from_instance(i2, pkg.configs.nvar(cfg))
        for _ in range(5):
            lev.coarse_step(-1.0)
        return shell_energy_np(oracle.assemble(lev, i2), i2)

    h = 1e-6
    errs = []
    for a, b, c in _directions(n, 3, 12):
        ct = torch.from_numpy(np.ascontiguousarray(c.transpose(2, 1, 0))).cuda()
        ad = dE * E0 * a + dR * R0 * b + float((dP * ct).sum())
        Jp = J_oracle(E0 * (1 + h * a), R0 * (1 + h * b), p["pert"] + h * c)
        Jm = J_oracle(E0 * (1 - h * a), R0 * (1 - h * b), p["pert"] - h * c)
        fd = (Jp - Jm) / (2 * h)
        errs.append(abs(ad - fd) / max(abs(ad), abs(fd)))
    print("oracle directional rel errors", ["%.2e" % e for e in errs])
    assert max(errs) <= 1e-5, errs
    run.close()


def test_autograd_function(pkg, table):
    import torch

    run, inst = _runner(pkg, table, 4, 4, 2)
    p = inst["problem"]
    E = torch.tensor(p["exp_energy"], dtype=torch.float64, requires_grad=True)
    R = torch.tensor(p["dens_ambient"], dtype=torch.float64, requires_grad=True)
    P = run.pert.clone().requires_grad_(True)
    J = pkg.adjoint.shell_energy(E, R, P, run)
    J.backward()
    # a second reverse sweep of the same forward: FP64 atomics reorder the
    # scatter sums, so the two agree to rounding, not bit for bit
    dE, dR, dP = run.backward()
    assert float(E.grad) == pytest.approx(dE, rel=1e-8)
    assert float(R.grad) == pytest.approx(dR, rel=1e-8)
    torch.testing.assert_close(P.grad, dP, rtol=1e-8, atol=1e-8 * float(dP.abs().max()))
    # one finite-difference direction through the Function itself
    h = 1e-6
    with torch.no_grad():
        Jp = pkg.adjoint.shell_energy(E * (1 + h), R, P, run)
        Jm = pkg.adjoint.shell_energy(E * (1 - h), R, P, run)
    fd = float(Jp - Jm) / (2 * h)
    assert fd == pytest.approx(float(E.grad) * float(E), rel=1e-5)
    run.close()


def _fd_steps(run, E0, R0, pert0, a, b, ct, steps=(1e-5, 1e-6, 1e-7)):
    out = []
    for h in steps:
        Jp = run.forward(E0 * (1 + h * a), R0 * (1 + h * b), pert0 + h * ct)
        Jm = run.forward(E0 * (1 - h * a), R0 * (1 - h * b), pert0 - h * ct)
        out.append((Jp - Jm) / (2 * h))
    return out


def test_gradient_converged_directions_c4(pkg, table):
    """The gradient configuration at its own size (64^3, 20 steps, checkpoint 5):
    along each of 16 seeded directions -- the blast energy alone, the ambient
    density alone, and 14 random combinations of both with the per-zone
    perturbation field -- the central finite difference is taken at relative
    steps 1e-5, 1e-6 and 1e-7.  Where those agree with each other to 1e-7 the
    finite difference has converged (no limiter or Riemann-sampling branch
    switch inside its stencil), and there the adjoint must match it to 1e-6;
    the other directions are reported with their spread."""
    import torch

    run, inst = _runner(pkg, table, 1, 20, 5)
    p = inst["problem"]
    E0, R0 = p["exp_energy"], p["dens_ambient"]
    pert0 = run.pert.clone()
    run.forward(E0, R0, pert0)
    dE, dR, dP = run.backward()
    n = run.n[0]
    zero = torch.zeros_like(pert0)
    dirs = [(1.0, 0.0, zero), (0.0, 1.0, zero)]
    for a, b, c in _directions(n, 14, 2019):
        dirs.append((a, b, torch.from_numpy(np.ascontiguousarray(c.transpose(2, 1, 0))).cuda()))
    converged, other = [], []
    for a, b, ct in dirs:
        ad = dE * E0 * a + dR * R0 * b + float((dP * ct).sum())
        f5, f6, f7 = _fd_steps(run, E0, R0, pert0, a, b, ct)
        scale = max(abs(f5), abs(f6), abs(f7))
        spread = max(abs(f5 - f6), abs(f6 - f7), abs(f5 - f7)) / scale
        err = abs(ad - f6) / max(abs(ad), abs(f6))
        (converged if spread <= 1e-7 else other).append((err, spread))
    print("converged directions (rel err, FD spread):", ["%.2e/%.1e" % e for e in converged])
    print("other directions (rel err, FD spread):", ["%.2e/%.1e" % e for e in other])
    assert converged, "no direction's finite difference converged"
    assert max(e for e, _ in converged) <= 1e-6, converged
    run.close()


def _rel(a, b):
    import torch

    if isinstance(a, torch.Tensor):
        return float((a - b).abs().max() / max(float(b.abs().max()), 1e-300))
    return abs(a - b) / max(abs(b), 1e-300)


def test_slab_reverse_matches_single_box(pkg, table):
    """The step reversed slab by slab (z-slabs of 8 zones of a 32^3 domain, each
    recomputing its forward with its own ghost zones and adding its Sborder
    adjoint into the domain's) gives the gradient the whole-domain reverse gives,
    to 1e-12: the full run from initdata (dJ/dE, dJ/drho, dJ/dpert) and a window
    of the last 4 of 8 steps (dJ/dV at step 4).  The forward is the same work
    zone by zone, so J is bit for bit the same."""
    K = pkg.castro
    L = K.init(*pkg.configs.NET2, table)
    cfg = pkg.configs.adjoint64(scale=2, steps=8)
    inst = cfg["instances"][0]
    p = inst["problem"]
    for first in (0, 4):
        out = []
        for slab in (0, 8):
            run = pkg.adjoint.SedovAdjoint(L, inst, 8, 3, cfg["shell"], slab_nz=slab, first_step=first)
            J = run.forward(p["exp_energy"], p["dens_ambient"])
            dE, dR, dP = run.backward()
            out.append((J, dE, dR, dP.clone(), run.state_adjoint()))
            run.close()
        (J0, dE0, dR0, dP0, V0), (J1, dE1, dR1, dP1, V1) = out
        assert J1 == J0
        assert _rel(V1, V0) <= 1e-12, f"window from step {first}: dJ/dV differs by {_rel(V1, V0):.2e}"
        if first == 0:
            assert _rel(dE1, dE0) <= 1e-12 and _rel(dR1, dR0) <= 1e-12 and _rel(dP1, dP0) <= 1e-12
        else:
            assert dE1 == 0.0 and dR1 == 0.0
        assert float(V0.abs().max()) > 0.0
