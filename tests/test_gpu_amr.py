"""The AMR pieces: flux register (crse_init, fine_add, reflux) and average_down.

* each kernel against a numpy statement of the same rule on random data;
* a two-level step with the library's own hydro: a periodic 16^3 coarse level
  (the reference problem's constants, 13 species) with a fine patch over its
  central 8^3 zones refined by 2, both advanced by one step of the same dt
  through castro_construct_hydro_source_box (fluxes out in store_flux's
  form), the fine ghost zones filled from the coarse state by injection; after
  average_down onto the coarse zones under the patch and reflux of the six
  faces of the patch, the coarse level's mass, momenta, total energy and
  species are conserved to round-off, which they are not without the reflux.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_harness import from_dev, sborder_from_domain, to_dev

pytestmark = pytest.mark.gpu


def _lib(pkg, table):
    A, Z = pkg.configs.NET13
    return pkg.castro.init(A, Z, table)


def _v(K, x):
    return K.ivec(x)


def test_average_down_matches_numpy(pkg, table):
    import torch

    L = _lib(pkg, table)
    K = pkg.castro
    rng = np.random.default_rng(5)
    r, nc = 2, 3
    clo, chi = (2, 3, 1), (9, 8, 6)
    flo, fhi = tuple(r * c for c in clo), tuple(r * h + r - 1 for h in chi)
    fine = np.asfortranarray(rng.standard_normal(tuple(h - l + 1 for l, h in zip(flo, fhi)) + (nc,)))
    crse = torch.zeros((nc,) + tuple(h - l + 1 for l, h in reversed(list(zip(clo, chi)))), dtype=torch.float64,
                       device="cuda")
    L.castro_average_down(_v(K, clo), _v(K, chi), C.c_void_p(crse.data_ptr()), _v(K, clo), _v(K, chi),
                          C.c_void_p(to_dev(fine).data_ptr()), _v(K, flo), _v(K, fhi), nc, r)
    torch.cuda.synchronize()
    K.check(L, "castro_average_down")
    shp = tuple(h - l + 1 for l, h in zip(clo, chi))
    # fine index r * I + a: in Fortran order the sub-index a varies fastest
    ref = fine.reshape(r, shp[0], r, shp[1], r, shp[2], nc, order="F").mean(axis=(0, 2, 4))
    np.testing.assert_allclose(from_dev(crse), ref, rtol=1e-15, atol=1e-15)


def test_amr_calls_reject_boxes_outside_their_arrays(pkg, table):
    import torch

    L = _lib(pkg, table)
    K = pkg.castro
    clo, chi = (0, 0, 0), (3, 3, 3)
    crse = torch.zeros((2, 4, 4, 4), dtype=torch.float64, device="cuda")
    fine = torch.ones((2, 7, 8, 8), dtype=torch.float64, device="cuda")   # one fine zone short along x
    L.castro_clear_error()
    L.castro_average_down(_v(K, clo), _v(K, chi), C.c_void_p(crse.data_ptr()), _v(K, clo), _v(K, chi),
                          C.c_void_p(fine.data_ptr()), _v(K, (0, 0, 0)), _v(K, (6, 7, 7)), 2, 2)
    assert L.castro_last_error() == 5 and b"outside" in L.castro_error_string()
    L.castro_clear_error()
    reg = torch.zeros((2, 4, 4, 1), dtype=torch.float64, device="cuda")
    L.castro_flux_register_reflux(_v(K, (0, 0, 0)), _v(K, (0, 3, 3)), 0, 0, C.c_void_p(crse.data_ptr()), _v(K, clo),
                                  _v(K, chi), C.c_void_p(reg.data_ptr()), _v(K, (0, 0, 0)), _v(K, (0, 3, 3)), 2,
                                  C.c_double(1.0))   # side 0 of face plane 0: the zones at x = -1
    assert L.castro_last_error() == 5
    L.castro_clear_error()
    torch.cuda.synchronize()
    assert float(crse.abs().max()) == 0.0      # nothing was launched


@pytest.mark.parametrize("d", [0, 1, 2])
def test_flux_register_matches_numpy(pkg, table, d):
    import torch

    L = _lib(pkg, table)
    K = pkg.castro
    rng = np.random.default_rng(10 + d)
    r, nc, vol = 2, 4, 0.125
    # coarse faces: one plane (normal d) of a patch face, 6 x 5 across
    flo = [3, 4, 5]
    fhi = [8, 8, 9]
    fhi[d] = flo[d]
    fb = tuple(h - l + 1 for l, h in zip(flo, fhi))
    crse_flux = np.asfortranarray(rng.standard_normal(fb + (nc,)))
    fflo = [r * x for x in flo]
    ffhi = [r * h + r - 1 for h in fhi]
    ffhi[d] = fflo[d]
    fine_flux = np.asfortranarray(rng.standard_normal(tuple(h - l + 1 for l, h in zip(fflo, ffhi)) + (nc,)))
    reg = torch.empty((nc,) + fb[::-1], dtype=torch.float64, device="cuda")
    L.castro_flux_register_crse_init(_v(K, flo), _v(K, fhi), C.c_void_p(reg.data_ptr()), _v(K, flo), _v(K, fhi),
                                     C.c_void_p(to_dev(crse_flux).data_ptr()), _v(K, flo), _v(K, fhi), nc)
    ff = to_dev(fine_flux)
    for _ in range(2):   # two fine substeps
        L.castro_flux_register_fine_add(_v(K, flo), _v(K, fhi), d, C.c_void_p(reg.data_ptr()), _v(K, flo),
                                        _v(K, fhi), C.c_void_p(ff.data_ptr()), _v(K, fflo), _v(K, ffhi), nc, r)
    torch.cuda.synchronize()
    K.check(L, "flux register")
    # numpy: the sum over each coarse face's r x r fine faces, twice, minus the coarse flux
    shp = list(fb)
    shp2 = []
    for a in range(3):
        shp2 += [1 if a == d else r, shp[a]]
    fsum = fine_flux.reshape(tuple(shp2) + (nc,), order="F").sum(axis=(0, 2, 4))
    ref = 2.0 * fsum - crse_flux
    got = from_dev(reg)
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=1e-14)
    # reflux onto both sides of the face plane
    slo = [l - 1 for l in flo]
    shi = [h + 1 for h in fhi]
    state0 = np.asfortranarray(rng.standard_normal(tuple(h - l + 1 for l, h in zip(slo, shi)) + (nc,)))
    for side in (0, 1):
        st = to_dev(state0)
        L.castro_flux_register_reflux(_v(K, flo), _v(K, fhi), d, side, C.c_void_p(st.data_ptr()), _v(K, slo),
                                      _v(K, shi), C.c_void_p(reg.data_ptr()), _v(K, flo), _v(K, fhi), nc,
                                      C.c_double(vol))
        torch.cuda.synchronize()
        K.check(L, "reflux")
        exp = state0.copy(order="F")
        sl = [slice(flo[a] - slo[a], fhi[a] - slo[a] + 1) for a in range(3)]
        if side == 0:
            sl[d] = slice(flo[d] - 1 - slo[d], flo[d] - slo[d])
            exp[tuple(sl)] -= ref / vol
        else:
            exp[tuple(sl)] += ref / vol
        np.testing.assert_allclose(from_dev(st), exp, rtol=1e-14, atol=1e-13)


def _hydro(L, K, lo, hi, sb, sblo, sbhi, nv, dx, dt):
    """castro_construct_hydro_source_box on one box: (source, [dt*F*A per direction])."""
    import torch

    src = torch.zeros((nv,) + tuple(h - l + 1 for l, h in reversed(list(zip(lo, hi)))), dtype=torch.float64,
                      device="cuda")
    fo, flos, fhis = [], [], []
    for d in range(3):
        h = list(hi)
        h[d] += 1
        flos += list(lo)
        fhis += h
        fo.append(torch.zeros((nv,) + tuple(b - a + 1 for a, b in reversed(list(zip(lo, h)))), dtype=torch.float64,
                              device="cuda"))
    ptrs = (C.c_void_p * 3)(*[f.data_ptr() for f in fo])
    K.call(L, "castro_clean_state", list(sblo), list(sbhi), sb, list(sblo), list(sbhi))
    rc = L.castro_construct_hydro_source_box(K.ivec(lo), K.ivec(hi), C.c_void_p(sb.data_ptr()), K.ivec(sblo),
                                             K.ivec(sbhi), C.c_void_p(src.data_ptr()), K.ivec(lo), K.ivec(hi), ptrs,
                                             (C.c_int * 9)(*flos), (C.c_int * 9)(*fhis), K.ivec(lo), K.ivec(hi),
                                             K.dvec(dx), C.c_double(dt))
    torch.cuda.synchronize()
    assert rc == 0, L.castro_error_string()
    return src, fo


def _two_level_step(pkg, table, do_reflux):
    import torch

    cfg = pkg.configs.reference(scale=8, max_box=64)   # 16^3, 13 species, periodic
    L = pkg.castro.init(*cfg["network"], table)
    K = pkg.castro
    nv = pkg.configs.nvar(cfg)
    sim = pkg.make_sim(L, cfg, K.MODE_BATCHED)
    sim.init_data()
    sim.step(3)
    inst = cfg["instances"][0]
    Gc = K.assemble(inst, sim.box_states()[0])
    dt = 0.5 * sim.est_time_step()          # the fine level's CFL with the coarse dt
    sim.close()
    n, r = 16, 2
    dxc = (inst["probhi"][0] - inst["problo"][0]) / n
    dxf = dxc / r
    vc = dxc ** 3
    plo, phi = (4, 4, 4), (11, 11, 11)     # coarse zones under the patch
    # fine level: injection of the coarse state onto the patch and its ghost zones
    flo, fhi = tuple(r * x for x in plo), tuple(r * h + r - 1 for h in phi)
    fsblo, fsbhi = tuple(x - 4 for x in flo), tuple(x + 4 for x in fhi)
    idx = [np.floor_divide(np.arange(fsblo[a], fsbhi[a] + 1), r) % n for a in range(3)]
    Fsb = np.asfortranarray(Gc[np.ix_(idx[0], idx[1], idx[2])])
    Uf0 = np.asfortranarray(Fsb[4:-4, 4:-4, 4:-4])
    # coarse step over the whole (periodic) domain as one box
    lo, hi = (0, 0, 0), (n - 1, n - 1, n - 1)
    csb = to_dev(sborder_from_domain(Gc, inst["dom_lo"], lo, hi, inst["bc"]))
    src_c, fo_c = _hydro(L, K, lo, hi, csb, (-4, -4, -4), (n + 3,) * 3, nv, [dxc] * 3, dt)
    Uc = to_dev(Gc)
    Uc += dt * src_c
    # fine step
    fsb = to_dev(Fsb)
    src_f, fo_f = _hydro(L, K, flo, fhi, fsb, fsblo, fsbhi, nv, [dxf] * 3, dt)
    Uf = to_dev(Uf0) + dt * src_f
    # average down onto the coarse zones under the patch
    L.castro_average_down(K.ivec(plo), K.ivec(phi), C.c_void_p(Uc.data_ptr()), K.ivec(lo), K.ivec(hi),
                          C.c_void_p(Uf.data_ptr()), K.ivec(flo), K.ivec(fhi), nv, r)
    if do_reflux:
        for d in range(3):
            for side, face in ((0, plo[d]), (1, phi[d] + 1)):
                # coarse faces of this side of the patch (coarse face indices), and the fine faces on them
                cflo, cfhi = list(plo), list(phi)
                cflo[d] = cfhi[d] = face
                ffl, ffh = [r * x for x in cflo], [r * h + r - 1 for h in cfhi]
                ffl[d] = ffh[d] = r * face
                reg = torch.empty((nv,) + tuple(h - l + 1 for l, h in reversed(list(zip(cflo, cfhi)))),
                                  dtype=torch.float64, device="cuda")
                clf, chf = list(lo), list(hi)
                chf[d] += 1
                L.castro_flux_register_crse_init(K.ivec(cflo), K.ivec(cfhi), C.c_void_p(reg.data_ptr()), K.ivec(cflo),
                                                 K.ivec(cfhi), C.c_void_p(fo_c[d].data_ptr()), K.ivec(clf),
                                                 K.ivec(chf), nv)
                fl, fh = list(flo), list(fhi)
                fh[d] += 1
                L.castro_flux_register_fine_add(K.ivec(cflo), K.ivec(cfhi), d, C.c_void_p(reg.data_ptr()),
                                                K.ivec(cflo), K.ivec(cfhi), C.c_void_p(fo_f[d].data_ptr()),
                                                K.ivec(fl), K.ivec(fh), nv, r)
                # side 0: the patch lies above the face, the coarse zone to correct below it
                L.castro_flux_register_reflux(K.ivec(cflo), K.ivec(cfhi), d, side, C.c_void_p(Uc.data_ptr()),
                                              K.ivec(lo), K.ivec(hi), C.c_void_p(reg.data_ptr()), K.ivec(cflo),
                                              K.ivec(cfhi), nv, C.c_double(vc))
    torch.cuda.synchronize()
    K.check(L, "two-level step")
    # the coarse level before the step, with the patch's zones averaged down from the fine
    # initial data (injection: the same values)
    return Gc, from_dev(Uc), vc


def test_two_level_reflux_conserves(pkg, table):
    G0, G1, vc = _two_level_step(pkg, table, True)
    comps = [0, 1, 2, 3, 4] + list(range(7, G0.shape[3]))     # rho, momenta, rho E, species
    for c in comps:
        a, b = G0[..., c].sum() * vc, G1[..., c].sum() * vc
        scale = np.abs(G0[..., c]).sum() * vc
        assert abs(b - a) <= 1e-12 * scale, (c, a, b)
    # without the reflux the coarse fluxes through the patch's faces and the fine ones disagree
    G0n, G1n, _ = _two_level_step(pkg, table, False)
    drift = abs(G1n[..., 0].sum() - G0n[..., 0].sum()) / np.abs(G0n[..., 0]).sum()
    assert drift > 1e-10, drift
