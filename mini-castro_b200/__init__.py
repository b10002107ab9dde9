"""mini-castro_b200: B200-native CTU hydro advance of mini-Castro.

The product is the CUDA library ``lib/libcastro_b200.so`` (C-ABI in
``include/castro_b200.h``); this package is its Python host side:

* ``castro``     -- ctypes binding of the C-ABI (simulation objects, per-routine calls)
* ``configs``    -- the Sedov workloads (BoxArrays, networks, problem constants)
* ``helm_table`` -- writer of the Helmholtz table file read by ``eos_init`` (analytic non-degenerate gas)
* ``helm_fd``    -- the same file computed from Fermi-Dirac integrals (electron-positron gas in pair equilibrium)
* ``replicas``   -- the multi-GPU (one replica per rank) reductions
* ``shard``      -- one level's boxes sharded over ranks: halo exchange, dt min-reduction
* ``adjoint``    -- gradients of a Sedov run (reverse sweep) and its torch.autograd wrapper
* ``plotfile``   -- reader of the AMReX plotfiles the library writes
* ``build``      -- nvcc recipe for the sm_100a libraries
"""
from . import adjoint, castro, configs, helm_fd, helm_table, plotfile, replicas, shard  # noqa: F401

__all__ = ["adjoint", "castro", "configs", "helm_fd", "helm_table", "plotfile", "replicas", "shard", "make_sim"]


def make_sim(L, cfg, mode=castro.MODE_BATCHED):
    """A castro.Sim for a workload from ``configs``; perturbation fields are
    uploaded to the device (torch is used only to hold device memory)."""
    import torch

    keep = []
    insts = []
    for inst in cfg["instances"]:
        p = dict(inst["problem"])
        pert = p.pop("pert", None)
        kw = {k: v for k, v in p.items() if k != "pert_amp"}
        prob = castro.make_problem(L, **kw)
        if pert is not None:
            t = torch.from_numpy(pert.transpose(2, 1, 0).copy()).cuda()   # Fortran order on the device
            keep.append(t)
            prob.pert = t.data_ptr()
            for d in range(3):
                prob.pert_lo[d] = inst["dom_lo"][d]
                prob.pert_hi[d] = inst["dom_hi"][d]
            prob.pert_amp = p["pert_amp"]
        i2 = dict(inst)
        i2["problem"] = prob
        insts.append(i2)
    sim = castro.Sim(L, insts, mode)
    sim._pert = keep
    return sim
