"""One level's BoxArray sharded over ranks: the reference's MPI domain
decomposition (AMReX DistributionMapping of the boxes over ranks, the
FillBoundary halo exchange inside FillPatch of Sborder,
Source/Castro_advance.cpp:62, and ParallelDescriptor::ReduceRealMin of the
CFL time step, Source/Castro.cpp:210), rebuilt on torch.distributed (NCCL
between GPUs, gloo on CPU).

* ``distribute``  -- owner rank of every box: contiguous runs of the BoxArray,
  balanced by zone count (the configs' BoxArrays are ordered z-slab by z-slab,
  so each rank holds slabs and exchanges only with its neighbours).
* ``FillPlan``    -- for every box, where each zone of its grow(box, 4) Sborder
  comes from (a zone of some box after the periodic wrap or the outflow clamp
  of the boundary condition), split into the copies a rank makes from its own
  boxes and one message per peer.  Every rank builds the same plan from the
  global BoxArray, so a sender's packing order is its receiver's unpacking
  order without any index exchange.
* ``ShardedLevel`` -- Castro::advance over the boxes this rank owns
  (clean_state(S_old), FillPatch with the halo exchange, clean_state(Sborder),
  construct_hydro_source per box, Saxpy, clean_state(S_new) and the
  post_timestep clean, Source/Castro_advance.cpp:32-97, Source/Castro.cpp:369)
  with computeNewDt on the all-reduced minimum of every rank's estdt
  (Source/Castro.cpp:175-295).  The per-box work goes through a kernels
  object; ``GpuKernels`` drives the library's per-routine C-ABI
  (Source/Castro_F.H entry points and castro_construct_hydro_source_box) on
  this rank's GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import castro

NG = 4          # ghost zones of Sborder, Source/Castro_advance.cpp:37
CFL = 0.5       # Source/Castro.cpp:212


def npts(lo, hi) -> int:
    return int(np.prod([h - l + 1 for l, h in zip(lo, hi)]))


def grow(lo, hi, g):
    return tuple(l - g for l in lo), tuple(h + g for h in hi)


def distribute(boxes, nranks: int) -> list[int]:
    """Owner rank of each box: contiguous runs of the BoxArray order with about
    equal zone counts (a rank gets at least one box while boxes remain)."""
    sizes = [npts(lo, hi) for lo, hi in boxes]
    total = float(sum(sizes))
    owner, acc, r = [], 0.0, 0
    for b, s in enumerate(sizes):
        left = len(boxes) - b
        if r < nranks - 1 and (acc + 0.5 * s > total * (r + 1) / nranks or left <= nranks - 1 - r) and acc > 0:
            r += 1
        owner.append(r)
        acc += s
    return owner


@dataclass
class Piece:
    """Zones of one box's Sborder that come from one source rank: the source
    boxes and their zone indices, and the Sborder indices they fill."""
    dst_box: int
    src_box: np.ndarray
    src_idx: np.ndarray
    dst_idx: np.ndarray


class FillPlan:
    """Where every zone of every box's grow(box, NG) comes from."""

    def __init__(self, boxes, dom_lo, dom_hi, bc: int, ng: int = NG):
        self.boxes = [(tuple(l), tuple(h)) for l, h in boxes]
        shape = tuple(h - l + 1 for l, h in zip(dom_lo, dom_hi))
        owner = np.full(shape, -1, dtype=np.int64)
        for b, (lo, hi) in enumerate(self.boxes):
            sl = tuple(slice(l - d, h - d + 1) for l, h, d in zip(lo, hi, dom_lo))
            if (owner[sl] >= 0).any():
                raise ValueError("boxes overlap")
            owner[sl] = b
        if (owner < 0).any():
            raise ValueError("boxes do not cover the domain")
        self.src = []   # per box: (source box, source zone index, Sborder index), Sborder in x-fastest order
        for lo, hi in self.boxes:
            glo, ghi = grow(lo, hi, ng)
            axes = []
            for d in range(3):
                r = np.arange(glo[d], ghi[d] + 1) - dom_lo[d]
                n = shape[d]
                r = np.mod(r, n) if bc == castro.BC_PERIODIC else np.clip(r, 0, n - 1)
                axes.append(r)
            # x fastest: index = i + nx * (j + ny * k)
            kk, jj, ii = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
            ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
            sb = owner[ii, jj, kk]
            blo = np.array([self.boxes[s][0] for s in range(len(self.boxes))])
            bhi = np.array([self.boxes[s][1] for s in range(len(self.boxes))])
            bn = bhi - blo + 1
            li = ii + dom_lo[0] - blo[sb, 0]
            lj = jj + dom_lo[1] - blo[sb, 1]
            lk = kk + dom_lo[2] - blo[sb, 2]
            sidx = li + bn[sb, 0] * (lj + bn[sb, 1] * lk)
            self.src.append((sb, sidx, np.arange(sb.size)))

    def pieces(self, owner: list[int], dst_rank: int, src_rank: int) -> list[Piece]:
        """The zones of dst_rank's Sborders that src_rank's boxes supply, box by
        box in BoxArray order, zones in Sborder order: the message src_rank packs
        and dst_rank unpacks (or dst_rank's own copies when they are equal)."""
        own = np.asarray(owner)
        out = []
        for b, (sb, sidx, didx) in enumerate(self.src):
            if owner[b] != dst_rank:
                continue
            m = own[sb] == src_rank
            if m.any():
                out.append(Piece(b, sb[m], sidx[m], didx[m]))
        return out


class GpuKernels:
    """The per-box work of Castro::advance through the library's C-ABI on
    device arrays (torch CUDA tensors holding Fortran-order FABs)."""

    CLEAN = ("enforce_minimum_density", "normalize_species", "reset_internal_e", "compute_temp")

    def __init__(self, L, nvar: int):
        import torch

        self.L, self.nvar, self.torch = L, nvar, torch
        self.dtbuf = torch.empty(1, dtype=torch.float64, device="cuda")

    def new(self, lo, hi):
        return self.torch.zeros(npts(lo, hi) * self.nvar, dtype=self.torch.float64, device="cuda")

    def clean(self, a, alo, ahi, lo, hi):
        # Castro::clean_state: the four routines of CLEAN in one launch (castro_clean_state)
        castro.call(self.L, "castro_clean_state", list(lo), list(hi), a, list(alo), list(ahi))

    def estdt(self, u, lo, hi, dx) -> float:
        self.dtbuf.fill_(1.79769313486231570e308)
        castro.call(self.L, "estdt", list(lo), list(hi), u, list(lo), list(hi), [float(x) for x in dx], self.dtbuf)
        return float(self.dtbuf.item())

    def hydro_source(self, sb, lo, hi, dom_lo, dom_hi, dx, dt):
        import ctypes as C

        src = self.new(lo, hi)
        glo, ghi = grow(lo, hi, NG)
        K = castro
        rc = self.L.castro_construct_hydro_source_box(
            K.ivec(lo), K.ivec(hi), C.c_void_p(sb.data_ptr()), K.ivec(glo), K.ivec(ghi), C.c_void_p(src.data_ptr()),
            K.ivec(lo), K.ivec(hi), None, None, None, K.ivec(dom_lo), K.ivec(dom_hi), K.dvec(dx), C.c_double(dt))
        if rc != 0:
            castro.check(self.L, "castro_construct_hydro_source_box")
        return src

    def saxpy(self, u, dt, src):
        import ctypes as C

        self.L.castro_saxpy(C.c_void_p(u.data_ptr()), C.c_void_p(src.data_ptr()), u.numel(), C.c_double(dt))
        castro.check(self.L, "castro_saxpy")

    def gather(self, a, idx):
        return a.view(self.nvar, -1)[:, self.torch.as_tensor(idx, device=a.device)]

    def scatter(self, a, idx, vals):
        a.view(self.nvar, -1)[:, self.torch.as_tensor(idx, device=a.device)] = vals

    def to_host(self, a):
        return a.cpu().numpy()

    def from_host(self, x):
        return self.torch.from_numpy(np.ascontiguousarray(x)).cuda()


class ShardedLevel:
    """The boxes of one instance that this rank owns, advanced in lockstep with
    the other ranks (one process per GPU; world 1 runs the whole level)."""

    def __init__(self, inst: dict, nvar: int, kernels, rank: int = 0, world: int = 1, group=None, device=None):
        self.inst, self.nvar, self.K = inst, nvar, kernels
        self.rank, self.world, self.group = rank, world, group
        self.device = device
        self.boxes = [(tuple(l), tuple(h)) for l, h in inst["boxes"]]
        self.owner = distribute(self.boxes, world)
        self.mine = [b for b, r in enumerate(self.owner) if r == rank]
        self.plan = FillPlan(self.boxes, inst["dom_lo"], inst["dom_hi"], inst["bc"])
        self.recv = {p: self.plan.pieces(self.owner, rank, p) for p in range(world)}     # p -> my Sborder zones
        self.send = {p: self.plan.pieces(self.owner, p, rank) for p in range(world) if p != rank}
        n = [h - l + 1 for l, h in zip(inst["dom_lo"], inst["dom_hi"])]
        self.dx = [(inst["probhi"][d] - inst["problo"][d]) / n[d] for d in range(3)]
        self.U = {}
        self.time, self.dt, self.steps = 0.0, 0.0, 0

    # -- state -------------------------------------------------------------
    def set_state(self, domain: np.ndarray):
        """This rank's boxes from a (nx, ny, nz, NVAR) domain array."""
        lo0 = self.inst["dom_lo"]
        for b in self.mine:
            lo, hi = self.boxes[b]
            sl = tuple(slice(l - d, h - d + 1) for l, h, d in zip(lo, hi, lo0))
            self.U[b] = self.K.from_host(np.asfortranarray(domain[sl]).ravel(order="F"))

    def box_state(self, b) -> np.ndarray:
        lo, hi = self.boxes[b]
        shape = tuple(h - l + 1 for l, h in zip(lo, hi)) + (self.nvar,)
        return self.K.to_host(self.U[b]).reshape(shape, order="F")

    # -- collectives ---------------------------------------------------------
    def _min_all(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())

    def fill_patch(self) -> dict:
        """Sborder of every box of this rank: own zones copied, the others
        received from their owners (FillBoundary's halo exchange)."""
        sb = {}
        for b in self.mine:
            glo, ghi = grow(*self.boxes[b], NG)
            sb[b] = self.K.new(glo, ghi)
        for pc in self.recv[self.rank]:
            for s in np.unique(pc.src_box):
                m = pc.src_box == s
                self.K.scatter(sb[pc.dst_box], pc.dst_idx[m], self.K.gather(self.U[int(s)], pc.src_idx[m]))
        if self.world > 1:
            import torch.distributed as dist

            reqs, inbox = [], {}
            for p, pcs in self.send.items():
                if not pcs:
                    continue
                parts = []
                for pc in pcs:
                    for s in np.unique(pc.src_box):
                        m = pc.src_box == s
                        parts.append(self.K.gather(self.U[int(s)], pc.src_idx[m]))
                buf = parts[0].new_empty((self.nvar, sum(x.shape[1] for x in parts)))
                o = 0
                for x in parts:
                    buf[:, o:o + x.shape[1]] = x
                    o += x.shape[1]
                reqs.append(dist.isend(buf.contiguous(), p, group=self.group))
            for p in range(self.world):
                if p == self.rank or not self.recv[p]:
                    continue
                n = sum(pc.dst_idx.size for pc in self.recv[p])
                ref = next(iter(sb.values()))
                inbox[p] = ref.new_empty((self.nvar, n))
                reqs.append(dist.irecv(inbox[p], p, group=self.group))
            for r in reqs:
                r.wait()
            for p, buf in inbox.items():
                o = 0
                for pc in self.recv[p]:
                    # the sender packed each piece source box by source box
                    for s in np.unique(pc.src_box):
                        m = pc.src_box == s
                        k = int(m.sum())
                        self.K.scatter(sb[pc.dst_box], pc.dst_idx[m], buf[:, o:o + k])
                        o += k
        return sb

    # -- the coarse step -------------------------------------------------------
    def est_time_step(self) -> float:
        est = 1.79769313486231570e308
        for b in self.mine:
            lo, hi = self.boxes[b]
            est = min(est, self.K.estdt(self.U[b], lo, hi, self.dx))
        return self._min_all(est) * CFL

    def coarse_step(self, stop_time: float = -1.0) -> float:
        """computeNewDt, Castro::advance and post_timestep's clean; returns dt."""
        if self.steps == 0:
            dt = 0.01 * self.est_time_step()                         # initialTimeStep, Castro.cpp:168-170
        else:
            dt = min(1.0e100, min(self.est_time_step(), 1.1e0 * self.dt))   # Castro.cpp:264-267
        eps = 0.001 * dt
        if stop_time >= 0.0 and (self.time + dt) > (stop_time - eps):
            dt = stop_time - self.time
        self.dt = dt
        for b in self.mine:                                          # clean_state(S_old), :51
            lo, hi = self.boxes[b]
            self.K.clean(self.U[b], lo, hi, lo, hi)
        sb = self.fill_patch()                                       # FillPatch(Sborder, 4), :62
        src = {}
        for b in self.mine:
            lo, hi = self.boxes[b]
            glo, ghi = grow(lo, hi, NG)
            self.K.clean(sb[b], glo, ghi, glo, ghi)                  # clean_state(Sborder), :66
        for b in self.mine:                                          # construct_hydro_source, :70
            lo, hi = self.boxes[b]
            src[b] = self.K.hydro_source(sb[b], lo, hi, self.inst["dom_lo"], self.inst["dom_hi"], self.dx, dt)
        for b in self.mine:
            lo, hi = self.boxes[b]
            self.K.saxpy(self.U[b], dt, src[b])                      # Saxpy, :74
            self.K.clean(self.U[b], lo, hi, lo, hi)                  # clean_state(S_new), :78
            self.K.clean(self.U[b], lo, hi, lo, hi)                  # post_timestep, Castro.cpp:369
        self.time += dt
        self.steps += 1
        return dt
