"""Gradients of a Sedov run through the castro_adj C-ABI.

``SedovAdjoint`` drives one instance (its domain advanced as one box on the
GPU): ``forward(E, rho_ambient, pert)`` runs initdata plus ``nsteps`` coarse
steps and returns the kinetic energy in the spherical shell
0.3 <= r/L <= 0.4 about the centre; ``backward()`` runs the checkpointed
reverse sweep and returns dJ/dE, dJ/drho_ambient and dJ/dpert (the per-zone
density perturbation field, rho = rho_ambient * (1 + pert_amp * pert)).

``SedovShellEnergy`` wraps the pair as a ``torch.autograd.Function`` so that
``torch.autograd`` (gradcheck, optimisers) can drive it.  torch only holds
device memory here; every computation is in the CUDA library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import castro


class SedovAdjoint:
    """slab_nz > 0 reverses each step slab by slab (z-slabs of slab_nz zones);
    first_step > 0 differentiates only steps first_step..nsteps-1, with respect
    to the state at first_step (``state_adjoint``)."""

    def __init__(self, L: C.CDLL, inst: dict, nsteps: int, checkpoint: int = 5, shell=(0.3, 0.4),
                 slab_nz: int = 0, first_step: int = 0):
        import torch

        self.L = L
        self.inst = inst
        self.nsteps = nsteps
        p = dict(inst["problem"])
        pert = p.pop("pert", None)
        self.pert_amp = float(p.pop("pert_amp", 0.0))
        self.prob_kw = p
        self.n = tuple(h - l + 1 for l, h in zip(inst["dom_lo"], inst["dom_hi"]))
        # the perturbation lives on the device in Fortran order: a C-order (nz, ny, nx) tensor
        if pert is None:
            pert = np.zeros(self.n)
            self.pert_amp = 0.0
        self.pert = torch.from_numpy(np.ascontiguousarray(pert.transpose(2, 1, 0))).cuda()
        desc = castro.InstanceDesc()
        for k in range(3):
            desc.dom_lo[k] = inst["dom_lo"][k]
            desc.dom_hi[k] = inst["dom_hi"][k]
            desc.problo[k] = inst["problo"][k]
            desc.probhi[k] = inst["probhi"][k]
        desc.bc = inst["bc"]
        one_lo = np.array(inst["dom_lo"], dtype=np.int32)
        one_hi = np.array(inst["dom_hi"], dtype=np.int32)
        self._keep = [one_lo, one_hi]
        desc.nbox = 1
        desc.box_lo = one_lo.ctypes.data_as(castro._ip)
        desc.box_hi = one_hi.ctypes.data_as(castro._ip)
        desc.prob = self._problem(p["exp_energy"], p["dens_ambient"])
        desc.stop_time = inst.get("stop_time", -1.0)
        self.h = L.castro_adj_create_window(C.byref(desc), nsteps, checkpoint, slab_nz, first_step)
        castro.check(L, "castro_adj_create")
        if not self.h:
            raise castro.CastroError("castro_adj_create returned NULL")
        L.castro_adj_set_shell(self.h, shell[0], shell[1])
        castro.check(L, "castro_adj_set_shell")

    def _problem(self, E: float, rho: float) -> castro.Problem:
        kw = dict(self.prob_kw)
        kw["exp_energy"] = float(E)
        kw["dens_ambient"] = float(rho)
        prob = castro.make_problem(self.L, **kw)
        prob.pert = self.pert.data_ptr()
        for d in range(3):
            prob.pert_lo[d] = self.inst["dom_lo"][d]
            prob.pert_hi[d] = self.inst["dom_hi"][d]
        prob.pert_amp = self.pert_amp
        return prob

    def close(self):
        if getattr(self, "h", None):
            self.L.castro_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, E: float, rho: float, pert=None) -> float:
        """J(E, rho_ambient, pert); pert: (nz, ny, nx) float64 CUDA tensor or None (keep)."""
        if pert is not None:
            self.pert.copy_(pert)
        prob = self._problem(E, rho)
        self.L.castro_adj_set_problem(self.h, C.byref(prob))
        castro.check(self.L, "castro_adj_set_problem")
        J = C.c_double()
        self.L.castro_adj_forward(self.h, C.byref(J))
        castro.check(self.L, "castro_adj_forward")
        return J.value

    def backward(self):
        """(dJ/dE, dJ/drho_ambient, dJ/dpert as a (nz, ny, nx) CUDA tensor)."""
        import torch

        dE, dr = C.c_double(), C.c_double()
        gp = torch.zeros_like(self.pert)
        self.L.castro_adj_backward(self.h, C.byref(dE), C.byref(dr), C.c_void_p(gp.data_ptr()))
        castro.check(self.L, "castro_adj_backward")
        torch.cuda.synchronize()
        return dE.value, dr.value, gp

    def state_adjoint(self):
        """dJ/dV at the window's first step as a C-order (NVAR, nz, ny, nx) CUDA tensor
        (after backward)."""
        import torch

        nv = 7 + castro_nspec(self.L)
        t = torch.empty((nv,) + self.n[::-1], dtype=torch.float64, device="cuda")
        self.L.castro_adj_initial_adjoint(self.h, C.c_void_p(t.data_ptr()))
        castro.check(self.L, "castro_adj_initial_adjoint")
        return t

    def dts(self) -> list[float]:
        return [self.L.castro_adj_dt(self.h, n) for n in range(self.nsteps)]

    def time_ms(self) -> tuple[float, float]:
        return self.L.castro_adj_time_ms(self.h, 0), self.L.castro_adj_time_ms(self.h, 1)

    def device_bytes(self) -> int:
        return int(self.L.castro_adj_device_bytes(self.h))

    def final_state(self):
        """Final state as a C-order (NVAR, nz, ny, nx) CUDA tensor."""
        import torch

        nv = 7 + castro_nspec(self.L)
        t = torch.empty((nv,) + self.n[::-1], dtype=torch.float64, device="cuda")
        self.L.castro_adj_final_state(self.h, C.c_void_p(t.data_ptr()))
        castro.check(self.L, "castro_adj_final_state")
        return t


def castro_nspec(L) -> int:
    return int(L.castro_nspec())


def _function():
    import torch

    class SedovShellEnergy(torch.autograd.Function):
        """J = SedovShellEnergy.apply(E, rho_ambient, pert, runner): E and
        rho_ambient are 0-d float64 tensors, pert a (nz, ny, nx) float64 CUDA
        tensor; runner a SedovAdjoint for the instance."""

        @staticmethod
        def forward(ctx, E, rho, pert, runner):
            ctx.runner = runner
            J = runner.forward(float(E), float(rho), pert.detach())
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            dE, dr, gp = ctx.runner.backward()
            g = float(gJ)
            return (torch.tensor(g * dE, dtype=torch.float64), torch.tensor(g * dr, dtype=torch.float64),
                    gp * g, None)

    return SedovShellEnergy


def shell_energy(E, rho, pert, runner):
    """Differentiable J(E, rho_ambient, pert) through the CUDA forward and adjoint."""
    return _function().apply(E, rho, pert, runner)
