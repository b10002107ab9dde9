"""Per-routine parity: every Source/Castro_F.H entry point of the library
against its oracle counterpart on identical inputs.

The oracle replays Castro::construct_hydro_source (Source/Castro_hydro.cpp:31-397)
on one box of a Sedov state advanced a few steps, keeping every intermediate
FAB.  Each GPU routine is then called through the C-ABI with the oracle's own
inputs of that routine, so a mismatch points at exactly one kernel.  Outputs
start as NaN on both sides, so values the reference never writes must stay
untouched.  The exact build must agree bit for bit; the production build
within RTOL_KERNEL (see gpu_harness).
"""
from __future__ import annotations

import numpy as np
import pytest

from gpu_harness import RTOL_EOS_DERIV, assert_match, from_dev, nan_dev, sborder_from_domain, to_dev

pytestmark = pytest.mark.gpu

_current = {}


def gpu_lib(pkg, table, network, exact):
    key = (exact, tuple(network[0]))
    L = pkg.castro.load(exact)
    if _current.get(exact) != key:
        pkg.castro.init(network[0], network[1], table, exact=exact)
        _current[exact] = key
    return L


def grow(lo, hi, g):
    return [l - g for l in lo], [h + g for h in hi]


def surround(lo, hi, d):
    h = list(hi)
    h[d] += 1
    return list(lo), h


def growv(lo, hi, v):
    return [l - x for l, x in zip(lo, v)], [h + x for h, x in zip(hi, v)]


class Case:
    """Oracle intermediates of construct_hydro_source for one box."""

    def __init__(self, oracle, pkg, table, cfg, steps, box):
        A, Z = cfg["network"]
        self.network = (A, Z)
        oracle.network_init(A, Z)
        oracle.eos_init(table)
        inst = cfg["instances"][0]
        nv = pkg.configs.nvar(cfg)
        self.nv, self.qv = nv, nv + 1
        lev, prob = oracle.level_from_instance(inst, nv)
        for _ in range(steps):
            lev.coarse_step(-1.0)
        self.dt = lev.est_time_step()
        G = oracle.assemble(lev, inst)
        lo, hi = inst["boxes"][box]
        self.lo, self.hi = list(lo), list(hi)
        self.dom_lo, self.dom_hi = list(inst["dom_lo"]), list(inst["dom_hi"])
        self.dx = [(inst["probhi"][d] - inst["problo"][d]) / (inst["dom_hi"][d] - inst["dom_lo"][d] + 1) for d in range(3)]
        self.problo, self.probhi = list(inst["problo"]), list(inst["probhi"])
        self.raw_valid = np.asfortranarray(G[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1])
        self.sb_lo, self.sb_hi = grow(lo, hi, 4)
        sb = sborder_from_domain(G, inst["dom_lo"], lo, hi, inst["bc"])
        self.rec = {}
        self.rec["sb_raw"] = sb.copy(order="F")
        self._run(oracle, sb)

    def _run(self, O, sb):
        lo, hi, nv, qv = self.lo, self.hi, self.nv, self.qv
        R = self.rec
        sl, sh = self.sb_lo, self.sb_hi
        # clean_state(Sborder), one routine at a time
        for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
            R[name + "_in"] = sb.copy(order="F")
            O.call(name, sl, sh, sb, sl, sh)
            R[name + "_out"] = sb.copy(order="F")
        R["sb"] = sb
        qlo, qhi = grow(lo, hi, 4)
        olo, ohi = grow(lo, hi, 1)
        self.qlo, self.qhi, self.olo, self.ohi = qlo, qhi, olo, ohi
        q = O.fab(qlo, qhi, qv)
        qa = O.fab(qlo, qhi, 4)
        O.call("ctoprim", qlo, qhi, sb, sl, sh, q, qlo, qhi, qa, qlo, qhi)
        R["q"], R["qaux"] = q, qa
        div = O.fab(olo, ohi, 1)
        O.call("divu", olo, ohi, q, qlo, qhi, self.dx, div, olo, ohi)
        R["div"] = div
        ebx = [surround(lo, hi, d) for d in range(3)]
        gebx = [grow(*ebx[d], 1) for d in range(3)]
        tg = {(0, 0): (0, 1, 1), (0, 1): (0, 0, 1), (0, 2): (0, 1, 0), (1, 0): (0, 0, 1), (1, 1): (1, 0, 1),
              (1, 2): (1, 0, 0), (2, 0): (0, 1, 0), (2, 1): (1, 0, 0), (2, 2): (1, 1, 0)}
        tbx = {k: growv(*ebx[k[0]], v) for k, v in tg.items()}
        self.ebx, self.gebx, self.tbx = ebx, gebx, tbx
        qm = {k: O.fab(*tbx[k], qv) for k in tbx}
        qp = {k: O.fab(*tbx[k], qv) for k in tbx}
        dt = self.dt
        for d in range(3):
            O.call("trace_ppm", olo, ohi, lo, hi, d + 1, q, qlo, qhi, qa, qlo, qhi, qm[d, d], *tbx[d, d],
                   qp[d, d], *tbx[d, d], self.dom_lo, self.dom_hi, self.dx, dt)
        R["qm_tr"] = {d: qm[d, d].copy(order="F") for d in range(3)}
        R["qp_tr"] = {d: qp[d, d].copy(order="F") for d in range(3)}
        hdtdx = [0.5 * dt / self.dx[d] for d in range(3)]
        cdtdx = [dt / self.dx[d] / 3.0 for d in range(3)]
        R["cf"], R["t1"], R["t2"] = [], [], []
        for d in range(3):
            t1, t2 = (1, 2) if d == 0 else (0, 2) if d == 1 else (0, 1)
            f1 = O.fab(olo, ohi, nv)
            qi = O.fab(olo, ohi, qv)
            g1 = O.fab(olo, ohi, 6)
            O.call("compute_flux", *tbx[d, d], qm[d, d], *tbx[d, d], qp[d, d], *tbx[d, d], f1, olo, ohi, qi, olo, ohi,
                   g1, olo, ohi, qa, qlo, qhi, d + 1)
            R["cf"].append(dict(box=tbx[d, d], ql=qm[d, d].copy(order="F"), qr=qp[d, d].copy(order="F"), flux=f1,
                                qint=qi, qg=g1, idir=d + 1))
            for t in (t1, t2):
                ins = (qm[t, t].copy(order="F"), qp[t, t].copy(order="F"))
                O.call("trans1", *tbx[t, d], d + 1, t + 1, qm[t, t], *tbx[t, t], qm[t, d], *tbx[t, d], qp[t, t],
                       *tbx[t, t], qp[t, d], *tbx[t, d], qa, qlo, qhi, f1, olo, ohi, g1, olo, ohi, cdtdx[d])
                R["t1"].append(dict(box=tbx[t, d], idir1=d + 1, idir2=t + 1, q2m=ins[0], q2p=ins[1], inbox=tbx[t, t],
                                    q2mo=qm[t, d].copy(order="F"), q2po=qp[t, d].copy(order="F"), f1=f1.copy(order="F"),
                                    q1=g1.copy(order="F"), cdtdx=cdtdx[d]))
        flux, qe = [], []
        for d in range(3):
            t1, t2 = (1, 2) if d == 0 else (0, 2) if d == 1 else (0, 1)
            f1, f2 = O.fab(olo, ohi, nv), O.fab(olo, ohi, nv)
            g1, g2 = O.fab(olo, ohi, 6), O.fab(olo, ohi, 6)
            qi = O.fab(olo, ohi, qv)
            O.call("compute_flux", *tbx[t1, t2], qm[t1, t2], *tbx[t1, t2], qp[t1, t2], *tbx[t1, t2], f1, olo, ohi, qi,
                   olo, ohi, g1, olo, ohi, qa, qlo, qhi, t1 + 1)
            O.call("compute_flux", *tbx[t2, t1], qm[t2, t1], *tbx[t2, t1], qp[t2, t1], *tbx[t2, t1], f2, olo, ohi, qi,
                   olo, ohi, g2, olo, ohi, qa, qlo, qhi, t2 + 1)
            ql, qr = O.fab(olo, ohi, qv), O.fab(olo, ohi, qv)
            O.call("trans2", *ebx[d], d + 1, t1 + 1, t2 + 1, qm[d, d], *tbx[d, d], ql, olo, ohi, qp[d, d], *tbx[d, d],
                   qr, olo, ohi, qa, qlo, qhi, f1, olo, ohi, f2, olo, ohi, g1, olo, ohi, g2, olo, ohi,
                   hdtdx[d], hdtdx[t1], hdtdx[t2])
            R["t2"].append(dict(box=ebx[d], dirs=(d + 1, t1 + 1, t2 + 1), qm=qm[d, d].copy(order="F"),
                                qp=qp[d, d].copy(order="F"), tb=tbx[d, d], f1=f1, f2=f2, g1=g1, g2=g2,
                                ql=ql.copy(order="F"), qr=qr.copy(order="F"), h=(hdtdx[d], hdtdx[t1], hdtdx[t2])))
            fx, qgd = O.fab(*gebx[d], nv), O.fab(*gebx[d], 6)
            O.call("compute_flux", *ebx[d], ql, olo, ohi, qr, olo, ohi, fx, *gebx[d], qi, olo, ohi, qgd, *gebx[d], qa,
                   qlo, qhi, d + 1)
            flux.append(fx)
            qe.append(qgd)
        R["flux_riemann"] = [f.copy(order="F") for f in flux]
        for d in range(3):
            O.call("apply_av", *ebx[d], d + 1, self.dx, div, olo, ohi, self.rec["sb"], self.sb_lo, self.sb_hi,
                   flux[d], *gebx[d])
        R["flux_av"] = [f.copy(order="F") for f in flux]
        for d in range(3):
            O.call("normalize_species_fluxes", *ebx[d], flux[d], *gebx[d])
        R["flux"] = flux
        R["qe"] = qe
        area = [self.dx[1] * self.dx[2], self.dx[0] * self.dx[2], self.dx[0] * self.dx[1]]
        R["area"] = [np.full(tuple(h - l + 1 for l, h in zip(*gebx[d])) + (1,), area[d], order="F") for d in range(3)]
        R["vol"] = np.full(tuple(h - l + 1 for l, h in zip(lo, hi)) + (1,), self.dx[0] * self.dx[1] * self.dx[2], order="F")
        src = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)) + (nv,), order="F")
        O.call("fill_hydro_source", lo, hi, self.rec["sb"], sl, sh, q, qlo, qhi, src, lo, hi,
               flux[0], *gebx[0], flux[1], *gebx[1], flux[2], *gebx[2], qe[0], *gebx[0], qe[1], *gebx[1], qe[2],
               *gebx[2], R["area"][0], *gebx[0], R["area"][1], *gebx[1], R["area"][2], *gebx[2], R["vol"], lo, hi,
               self.dx, dt)
        R["src"] = src


def _cases(oracle, pkg, table):
    return {
        "sedov_ns2": Case(oracle, pkg, table, pkg.configs.sedov64(scale=4), 3, 0),
        "reference_ns13": Case(oracle, pkg, table, pkg.configs.reference(scale=8, max_box=8), 3, 5),
    }


@pytest.fixture(scope="module")
def cases(oracle, pkg, table):
    return _cases(oracle, pkg, table)


PARAMS = [(c, e) for c in ("sedov_ns2", "reference_ns13") for e in (True, False)]
IDS = [f"{c}-{'exact' if e else 'fast'}" for c, e in PARAMS]


@pytest.fixture(params=PARAMS, ids=IDS)
def env(request, cases, pkg, table, oracle):
    name, exact = request.param
    C = cases[name]
    # the oracle's network is process-global: select this case's species set
    # before any oracle call of the test (array sizes depend on it)
    oracle.network_init(*C.network)
    L = gpu_lib(pkg, table, C.network, exact)
    return C, L, exact, pkg.castro


def test_clean_state_routines(env):
    C, L, exact, K = env
    for name in ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp"):
        t = to_dev(C.rec[name + "_in"])
        K.call(L, name, C.sb_lo, C.sb_hi, t, C.sb_lo, C.sb_hi)
        assert_match(from_dev(t), C.rec[name + "_out"], exact, what=name)


def test_castro_clean_state(env):
    """The coarse castro_clean_state (the four routines in one launch) against the
    oracle's four routines applied in turn, from the raw Sborder."""
    C, L, exact, K = env
    t = to_dev(C.rec["enforce_minimum_density_in"])
    K.call(L, "castro_clean_state", C.sb_lo, C.sb_hi, t, C.sb_lo, C.sb_hi)
    assert_match(from_dev(t), C.rec["compute_temp_out"], exact, what="castro_clean_state")


def test_ctoprim(env):
    C, L, exact, K = env
    q, qa = nan_dev(C.qlo, C.qhi, C.qv), nan_dev(C.qlo, C.qhi, 4)
    K.call(L, "ctoprim", C.qlo, C.qhi, to_dev(C.rec["sb"]), C.sb_lo, C.sb_hi, q, C.qlo, C.qhi, qa, C.qlo, C.qhi)
    assert_match(from_dev(q), C.rec["q"], exact, what="ctoprim q")
    assert_match(from_dev(qa), C.rec["qaux"], exact, rtol=RTOL_EOS_DERIV, what="ctoprim qaux")


def test_divu(env):
    C, L, exact, K = env
    div = nan_dev(C.olo, C.ohi, 1)
    K.call(L, "divu", C.olo, C.ohi, to_dev(C.rec["q"]), C.qlo, C.qhi, C.dx, div, C.olo, C.ohi)
    assert_match(from_dev(div), C.rec["div"], exact, what="divu")


def test_trace_ppm(env):
    C, L, exact, K = env
    q, qa = to_dev(C.rec["q"]), to_dev(C.rec["qaux"])
    for d in range(3):
        tb = C.tbx[d, d]
        qm, qp = nan_dev(*tb, C.qv), nan_dev(*tb, C.qv)
        K.call(L, "trace_ppm", C.olo, C.ohi, C.lo, C.hi, d + 1, q, C.qlo, C.qhi, qa, C.qlo, C.qhi, qm, *tb, qp, *tb,
               C.dom_lo, C.dom_hi, C.dx, C.dt)
        assert_match(from_dev(qm), C.rec["qm_tr"][d], exact, what=f"trace_ppm qm d={d}")
        assert_match(from_dev(qp), C.rec["qp_tr"][d], exact, what=f"trace_ppm qp d={d}")


def test_compute_flux(env):
    C, L, exact, K = env
    qa = to_dev(C.rec["qaux"])
    for r in C.rec["cf"]:
        f, qi, g = nan_dev(C.olo, C.ohi, C.nv), nan_dev(C.olo, C.ohi, C.qv), nan_dev(C.olo, C.ohi, 6)
        K.call(L, "compute_flux", *r["box"], to_dev(r["ql"]), *r["box"], to_dev(r["qr"]), *r["box"], f, C.olo, C.ohi,
               qi, C.olo, C.ohi, g, C.olo, C.ohi, qa, C.qlo, C.qhi, r["idir"])
        assert_match(from_dev(f), r["flux"], exact, what="compute_flux flux")
        assert_match(from_dev(g), r["qg"], exact, what="compute_flux qgdnv")
        assert_match(from_dev(qi), r["qint"], exact, what="compute_flux qint")


def test_trans1(env):
    C, L, exact, K = env
    qa = to_dev(C.rec["qaux"])
    for r in C.rec["t1"]:
        mo, po = nan_dev(*r["box"], C.qv), nan_dev(*r["box"], C.qv)
        K.call(L, "trans1", *r["box"], r["idir1"], r["idir2"], to_dev(r["q2m"]), *r["inbox"], mo, *r["box"],
               to_dev(r["q2p"]), *r["inbox"], po, *r["box"], qa, C.qlo, C.qhi, to_dev(r["f1"]), C.olo, C.ohi,
               to_dev(r["q1"]), C.olo, C.ohi, r["cdtdx"])
        assert_match(from_dev(mo), r["q2mo"], exact, what=f"trans1 {r['idir1']}->{r['idir2']} minus")
        assert_match(from_dev(po), r["q2po"], exact, what=f"trans1 {r['idir1']}->{r['idir2']} plus")


def test_trans2(env):
    C, L, exact, K = env
    qa = to_dev(C.rec["qaux"])
    for r in C.rec["t2"]:
        ql, qr = nan_dev(C.olo, C.ohi, C.qv), nan_dev(C.olo, C.ohi, C.qv)
        K.call(L, "trans2", *r["box"], *r["dirs"], to_dev(r["qm"]), *r["tb"], ql, C.olo, C.ohi, to_dev(r["qp"]),
               *r["tb"], qr, C.olo, C.ohi, qa, C.qlo, C.qhi, to_dev(r["f1"]), C.olo, C.ohi, to_dev(r["f2"]), C.olo,
               C.ohi, to_dev(r["g1"]), C.olo, C.ohi, to_dev(r["g2"]), C.olo, C.ohi, *r["h"])
        assert_match(from_dev(ql), r["ql"], exact, what=f"trans2 d={r['dirs'][0]} left")
        assert_match(from_dev(qr), r["qr"], exact, what=f"trans2 d={r['dirs'][0]} right")


def test_apply_av_and_normalize(env):
    C, L, exact, K = env
    div, sb = to_dev(C.rec["div"]), to_dev(C.rec["sb"])
    for d in range(3):
        f = to_dev(C.rec["flux_riemann"][d])
        K.call(L, "apply_av", *C.ebx[d], d + 1, C.dx, div, C.olo, C.ohi, sb, C.sb_lo, C.sb_hi, f, *C.gebx[d])
        assert_match(from_dev(f), C.rec["flux_av"][d], exact, what=f"apply_av d={d}")
        K.call(L, "normalize_species_fluxes", *C.ebx[d], f, *C.gebx[d])
        assert_match(from_dev(f), C.rec["flux"][d], exact, what=f"normalize_species_fluxes d={d}")


def test_fill_hydro_source(env):
    C, L, exact, K = env
    R = C.rec
    src = to_dev(np.zeros_like(R["src"]))
    g = C.gebx
    K.call(L, "fill_hydro_source", C.lo, C.hi, to_dev(R["sb"]), C.sb_lo, C.sb_hi, to_dev(R["q"]), C.qlo, C.qhi, src,
           C.lo, C.hi, to_dev(R["flux"][0]), *g[0], to_dev(R["flux"][1]), *g[1], to_dev(R["flux"][2]), *g[2],
           to_dev(R["qe"][0]), *g[0], to_dev(R["qe"][1]), *g[1], to_dev(R["qe"][2]), *g[2],
           to_dev(R["area"][0]), *g[0], to_dev(R["area"][1]), *g[1], to_dev(R["area"][2]), *g[2],
           to_dev(R["vol"]), C.lo, C.hi, C.dx, C.dt)
    assert_match(from_dev(src), R["src"], exact, what="fill_hydro_source")


def test_store_flux(env, oracle):
    C, L, exact, K = env
    for d in range(3):
        fo_ref = oracle.fab(*C.ebx[d], C.nv)
        oracle.call("store_flux", *C.ebx[d], fo_ref, *C.ebx[d], C.rec["flux"][d], *C.gebx[d], C.rec["area"][d],
                    *C.gebx[d], C.dt)
        fo = nan_dev(*C.ebx[d], C.nv)
        K.call(L, "store_flux", *C.ebx[d], fo, *C.ebx[d], to_dev(C.rec["flux"][d]), *C.gebx[d],
               to_dev(C.rec["area"][d]), *C.gebx[d], C.dt)
        assert_match(from_dev(fo), fo_ref, exact, what=f"store_flux d={d}")


def test_estdt(env, oracle):
    import torch

    C, L, exact, K = env
    ref = np.array([1.0e300])
    oracle.call("estdt", C.lo, C.hi, C.raw_valid, C.lo, C.hi, C.dx, ref)
    dt = torch.tensor([1.0e300], dtype=torch.float64, device="cuda")
    K.call(L, "estdt", C.lo, C.hi, to_dev(C.raw_valid), C.lo, C.hi, C.dx, dt)
    got = float(dt.item())
    if exact:
        assert got == ref[0]
    else:
        assert abs(got / ref[0] - 1) <= 1e-14


def test_initdata_and_diagnostics(env, oracle, pkg):
    import torch

    C, L, exact, K = env
    # the reference problem constants, installed on both sides
    if len(C.network[0]) == 13:
        kw = dict(ambient_from_T=0, dens_ambient=1e4, p_ambient=1e21, exp_energy=1e52, r_init=1.25e8, X=[1.0])
    else:
        kw = dict(ambient_from_T=1, dens_ambient=1.0, T_ambient=1e6, exp_energy=1e50, r_init=4 * C.dx[0], X=[0.5, 0.5])
    oracle.Problem(**kw).install()
    p = K.make_problem(L, **kw)
    L.castro_set_problem(K.C.byref(p))
    u_ref = oracle.fab(C.lo, C.hi, C.nv)
    oracle.call("initdata", C.lo, C.hi, u_ref, C.lo, C.hi, C.dx, C.problo, C.probhi)
    u = nan_dev(C.lo, C.hi, C.nv)
    K.call(L, "initdata", C.lo, C.hi, u, C.lo, C.hi, C.dx, C.problo, C.probhi)
    assert_match(from_dev(u), u_ref, exact, what="initdata")
    # blast-radius sums (order of the device atomics differs from the CPU loop)
    U = C.raw_valid
    maxd = float(U[..., 0].max())
    bm, br = np.zeros(1), np.zeros(1)
    oracle.call("calculate_blast_radius", C.lo, C.hi, U, C.lo, C.hi, C.dx, C.problo, C.probhi, bm, br, maxd)
    d2 = torch.zeros(2, dtype=torch.float64, device="cuda")
    K.call(L, "calculate_blast_radius", C.lo, C.hi, to_dev(U), C.lo, C.hi, C.dx, C.problo, C.probhi,
           K.C.c_void_p(d2.data_ptr()), K.C.c_void_p(d2.data_ptr() + 8), maxd)
    got = d2.cpu().numpy()
    np.testing.assert_allclose(got, [bm[0], br[0]], rtol=1e-13)
    # denerror tags
    den_lo, den_hi = grow(C.lo, C.hi, 1)
    den = np.asfortranarray(C.rec["sb_raw"][3:-3, 3:-3, 3:-3, 0])
    tag_ref = np.zeros(tuple(h - l + 1 for l, h in zip(C.lo, C.hi)), dtype=np.int8, order="F")
    oracle.call("denerror", C.lo, C.hi, tag_ref, C.lo, C.hi, den, den_lo, den_hi, 1, 0)
    tag = torch.zeros(tag_ref.size, dtype=torch.int8, device="cuda")
    K.call(L, "denerror", C.lo, C.hi, K.C.c_void_p(tag.data_ptr()), C.lo, C.hi, to_dev(den[..., None]), den_lo,
           den_hi, 1, 0)
    got_tag = tag.cpu().numpy().reshape(tag_ref.shape, order="F")
    np.testing.assert_array_equal(got_tag, tag_ref)
