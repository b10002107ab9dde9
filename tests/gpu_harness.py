"""Helpers of the GPU parity tests: oracle <-> device array transfer and the
comparison criteria.

Tolerances (FP64):
* exact build (-DCASTRO_EXACT --fmad=false): bit-for-bit equality with the oracle;
* production build, small cases: per component, max |gpu - oracle| /
  max(|oracle|, FLOOR * scale_c) <= RTOL_STEP after one step, where scale_c is
  the component's largest magnitude in the array, and relative L1 per component
  <= RTOL_L1 after a run;
* production build at the configurations' own sizes: the strict per-zone
  criterion below (no magnitude floor; round-off noise zones reported apart).
"""
from __future__ import annotations

import numpy as np
import torch

RTOL_KERNEL = 1e-12   # one routine on identical inputs
# EOS derivative outputs (gamma_1, dp/de, dp/drho|e): the production build
# contracts the biquintic table interpolation in a different order (a sum of
# 36 terms that cancel strongly in the derivative weights), so these agree
# to ~1e-12 rather than 1e-13; no hydro stage consumes dp/de or dp/drho|e.
RTOL_EOS_DERIV = 1e-11
RTOL_STEP = 1e-12     # state after one coarse step
RTOL_L1 = 1e-9        # relative L1 after a full run
FLOOR = 1e-3


def to_dev(a: np.ndarray) -> torch.Tensor:
    """Fortran-order (nx,ny,nz,nc) numpy array -> device buffer with the same memory layout."""
    if a.ndim == 3:
        a = a[..., None]
    return torch.from_numpy(np.ascontiguousarray(a.transpose(3, 2, 1, 0))).cuda()


def from_dev(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().transpose(3, 2, 1, 0)


def nan_dev(lo, hi, nc) -> torch.Tensor:
    shape = (nc,) + tuple(h - l + 1 for l, h in reversed(list(zip(lo, hi))))
    return torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")


def scaled_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per component: max over zones of |a-b| / max(|b|, FLOOR * max|b|); NaNs must coincide."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim == 3:
        a, b = a[..., None], b[..., None]
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN pattern differs (a value the reference never writes was produced or read)"
    nc = a.shape[-1]
    out = np.zeros(nc)
    for c in range(nc):
        ac, bc = a[..., c], b[..., c]
        m = ~np.isnan(bc)
        if not m.any():
            continue
        scale = np.abs(bc[m]).max()
        if scale == 0:
            out[c] = np.abs(ac[m]).max()
            continue
        den = np.maximum(np.abs(bc[m]), FLOOR * scale)
        out[c] = (np.abs(ac[m] - bc[m]) / den).max()
    return out


# Strict per-zone criterion of the configuration-size tests.  The relative
# error of a zone is |gpu - oracle| / max(|oracle|, TINY), TINY the smallest
# normal double: no floor tied to the component's magnitude.  A zone whose value
# is round-off noise -- the result of a cancellation, so that any other correct
# rounding of the same algorithm moves it far more than 1e-12 -- cannot meet a
# per-zone relative bar in a contracting build.  Such zones are identified
# without the GPU: the oracle's timing build (liboracle_fast.so: FMA contraction
# and the table interpolation summed in the production build's order) is run on
# the same inputs, and a zone it moves by more than NOISE_RTOL relative is noise;
# so is a zone whose one-step value is a cancellation (cancellation_mask: below
# CANCEL of the magnitude of the state and flux terms that formed it).  Noise
# zones are reported apart and must agree to NOISE_ABS of their component's
# largest magnitude; every other zone must meet RTOL_STEP.
TINY = float(np.finfo(np.float64).tiny)
NOISE_RTOL = 1e-14
NOISE_ABS = 1e-13


def noise_mask(ref: np.ndarray, contracted: np.ndarray) -> np.ndarray:
    """Zones (per component) whose value the contracting CPU build moves by more than NOISE_RTOL."""
    return np.abs(contracted - ref) > NOISE_RTOL * np.maximum(np.abs(ref), TINY)


CANCEL = 1e-3


def cancellation_mask(u_old: np.ndarray, u_new: np.ndarray, dt: float, dx: float) -> np.ndarray:
    """Zones (per component) whose value after one step is below CANCEL of the
    magnitude of the terms that formed it: U_new = U_old + dt * (flux difference)
    / dx, each face flux bounded by the old state of the zone and its six face
    neighbours -- rho|u| (density), rho u^2 + p (momenta), (E + p)|u|
    (total energy), (rho e + p)|u| + p|u| (internal energy, with p div u) --
    with p bounded by rho e (gamma - 1 <= 1).  Such a value is a cancellation:
    its relative rounding error is amplified by more than 1/CANCEL, so a
    per-zone relative bar of 1e-12 does not apply to it.  Only density, momenta
    and energies are flux balances: the temperature is an EOS output, and the
    species slots hold X after normalize_species (the reference divides rho X
    by its sum, Source/Castro_nd.F90:152-154), so neither is flagged here."""
    rho = u_old[..., 0]
    u = [u_old[..., 1 + d] / rho for d in range(3)]
    speed = np.abs(u[0]) + np.abs(u[1]) + np.abs(u[2])
    rhoe = np.abs(u_old[..., 5])
    p = rhoe
    scale = {0: rho * speed, 1: rho * speed * speed + p, 4: (np.abs(u_old[..., 4]) + p) * speed,
             5: (rhoe + p) * speed + p * speed}
    scale[2] = scale[3] = scale[1]

    def nbr_max(a):
        g = np.pad(a, 1, mode="edge")
        out = a.copy()
        for d in range(3):
            lo = [slice(1, -1)] * 3
            hi = [slice(1, -1)] * 3
            lo[d], hi[d] = slice(0, -2), slice(2, None)
            out = np.maximum(out, np.maximum(g[tuple(lo)], g[tuple(hi)]))
        return out

    mask = np.zeros(u_new.shape, dtype=bool)
    for c in range(6):
        f = scale[c]
        terms = np.abs(u_old[..., c]) + 6.0 * dt / dx * nbr_max(f)
        mask[..., c] = np.abs(u_new[..., c]) < CANCEL * terms
    return mask


def strict_zone_report(gpu: np.ndarray, ref: np.ndarray, noise: np.ndarray) -> list[dict]:
    """Per component: zones, noise zones, worst relative error over the other
    zones, worst |gpu - ref| / max|ref| over the noise zones."""
    nc = ref.shape[-1]
    A, B, N = gpu.reshape(-1, nc), ref.reshape(-1, nc), noise.reshape(-1, nc)
    out = []
    for c in range(nc):
        a, b, n = A[:, c], B[:, c], N[:, c]
        d = np.abs(a - b)
        with np.errstate(over="ignore"):
            rel = d / np.maximum(np.abs(b), TINY)
        scale = float(np.abs(b).max()) or 1.0
        out.append({"zones": int(b.size), "noise_zones": int(n.sum()),
                    "zones_above_rtol": int((rel > RTOL_STEP).sum()),
                    "max_rel": float(rel[~n].max()) if (~n).any() else 0.0,
                    "noise_max_abs_over_scale": float(d[n].max() / scale) if n.any() else 0.0})
    return out


def assert_strict(gpu: np.ndarray, ref: np.ndarray, noise: np.ndarray, what: str = "") -> list[dict]:
    rep = strict_zone_report(gpu, ref, noise)
    bad = [(c, r) for c, r in enumerate(rep) if r["max_rel"] > RTOL_STEP or r["noise_max_abs_over_scale"] > NOISE_ABS]
    assert not bad, f"{what}: per-zone check failed (component, report): {bad}"
    return rep


def assert_match(gpu: np.ndarray, ref: np.ndarray, exact: bool, rtol: float = RTOL_KERNEL, what: str = ""):
    if exact:
        np.testing.assert_array_equal(gpu, ref, err_msg=f"{what}: exact build must match the oracle bit for bit")
    else:
        e = scaled_err(gpu, ref)
        assert (e <= rtol).all(), f"{what}: scaled error {e.max():.3e} > {rtol:g} (per component {e})"


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    nc = a.shape[-1]
    A, B = a.reshape(-1, nc), b.reshape(-1, nc)
    num = np.abs(A - B).sum(0)
    den = np.abs(B).sum(0)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def sborder_from_domain(G: np.ndarray, dom_lo, lo, hi, bc: int, ng: int = 4) -> np.ndarray:
    """FillPatch of one box's Sborder (grow(box, ng)) from a domain array:
    periodic wrap (bc 0) or zero-gradient copy of the nearest zone (bc 1)."""
    idx = []
    for d in range(3):
        n = G.shape[d]
        r = np.arange(lo[d] - ng, hi[d] + ng + 1) - dom_lo[d]
        r = np.mod(r, n) if bc == 0 else np.clip(r, 0, n - 1)
        idx.append(r)
    return np.asfortranarray(G[np.ix_(idx[0], idx[1], idx[2])])
