"""z-slab decomposition of one domain over several ranks (one GPU each).

The reference decomposes its grid over MPI ranks (build_cart_decomp /
compute_local_desc, field_structures.h:1062-1115) and exchanges, per RK
stage, three ghost planes of the primitives (exchange_halos_physical,
field_structures.h:936-994), the half-node face fluxes
(exchange_halos_halfnode_flux, :998-1056) and the node viscous fluxes
(exchange_halos_viscous_flux, :877-932).  Here the domain is split along z
only, and each rank keeps HALO = 6 extra planes of primitives (and
temperature) on each side that borders another rank.  With six planes every
face flux and node viscous flux a rank's own cells need is computed locally
from identical inputs, so one exchange per stage -- the primitive halo --
replaces the reference's three, and the owned cells come out bit for bit
equal to a single-domain run:

  * a face flux reads cells i-2 .. i+3 and the 6th-order half-node
    difference of cell i reads faces i-5/2 .. i+5/2, so the owned cells need
    cells up to five planes beyond them;
  * a node viscous flux reads gradients over +-3 planes and the divergence
    of cell i reads node fluxes over +-3 planes: six planes.

The local handle treats a halo side as a non-periodic boundary; its
boundary treatment (ghost faces, reduced viscous orders) reaches three
planes into the halo, never an owned plane.  The x/y sweeps run only over
the owned planes, the viscous kernel over the owned planes and three halo
planes each side, the z-sweep updates only owned cells, and the CFL and
kinetic-energy reductions count only owned cells (ns3d_set_slab).

This module holds the host-side plan (which planes each rank owns, sends
and receives), the halo exchange over torch.distributed point-to-point
operations (NCCL between GPUs, gloo on the CPU), and ``SlabSolver``, the
per-rank driver over the C ABI.  No collective touches the field data
except the halo exchange; the time step is one MIN all-reduce of a double.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

HALO = 6


@dataclass(frozen=True)
class SlabPlan:
    """One rank's share of a z-decomposition of nz global planes."""
    nz: int                 # global interior planes
    world: int
    rank: int
    periodic: bool          # z periodic in the global problem
    z0: int                 # first owned global plane
    z1: int                 # one past the last owned global plane
    lower: Optional[int]    # rank holding the planes below (None: a real boundary)
    upper: Optional[int]    # rank holding the planes above

    @property
    def owned(self) -> int:
        return self.z1 - self.z0

    @property
    def halo_lo(self) -> int:
        return HALO if self.lower is not None else 0

    @property
    def halo_hi(self) -> int:
        return HALO if self.upper is not None else 0

    @property
    def nz_local(self) -> int:
        return self.owned + self.halo_lo + self.halo_hi

    @property
    def zlo(self) -> int:
        """First owned plane in local interior indices."""
        return self.halo_lo

    @property
    def zhi(self) -> int:
        return self.halo_lo + self.owned

    def global_planes(self) -> np.ndarray:
        """Global plane index of every local interior plane (wrapped when periodic)."""
        g = np.arange(self.z0 - self.halo_lo, self.z1 + self.halo_hi)
        return g % self.nz if self.periodic else g


def slab_plan(nz: int, world: int, rank: int, periodic: bool) -> SlabPlan:
    """Block distribution of the z-planes, the first nz % world ranks one
    plane larger (compute_local_desc's split, field_structures.h:1097-1115)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    base, extra = divmod(nz, world)
    sizes = [base + (1 if r < extra else 0) for r in range(world)]
    if world > 1 and min(sizes) < HALO:
        raise ValueError(f"each rank needs at least {HALO} owned z-planes (nz={nz}, world={world})")
    z0 = sum(sizes[:rank])
    z1 = z0 + sizes[rank]
    if world == 1:
        return SlabPlan(nz, 1, 0, periodic, 0, nz, None, None)
    lower = (rank - 1) % world if (rank > 0 or periodic) else None
    upper = (rank + 1) % world if (rank < world - 1 or periodic) else None
    return SlabPlan(nz, world, rank, periodic, z0, z1, lower, upper)


def exchange(plan: SlabPlan, planes: Callable[[str, int, int], Sequence], group=None) -> None:
    """The halo exchange of one stage over torch.distributed point-to-point
    operations, in two phases so that every pair of ranks has one send and
    one receive per phase (with two ranks and periodic z both neighbours are
    the same rank):
      phase 1: send the top HALO owned planes up, receive the lower halo from below;
      phase 2: send the bottom HALO owned planes down, receive the upper halo from above.
    planes(side, k0, count) returns the tensors (one per exchanged field) of
    local interior planes [k0, k0 + count)."""
    import torch.distributed as dist
    if plan.world == 1:
        return
    phases = [(plan.upper, plan.zhi - HALO, plan.lower, plan.zlo - HALO),
              (plan.lower, plan.zlo, plan.upper, plan.zhi)]
    for send_to, send_k0, recv_from, recv_k0 in phases:
        ops = []
        if recv_from is not None:
            for t in planes("recv", recv_k0, HALO):
                ops.append(dist.P2POp(dist.irecv, t, recv_from, group))
        if send_to is not None:
            for t in planes("send", send_k0, HALO):
                ops.append(dist.P2POp(dist.isend, t, send_to, group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()


class _DeviceArray:
    """A raw device range as a torch tensor (via __cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def device_planes(solver, k0: int, count: int) -> List:
    """Tensors viewing local interior planes [k0, k0 + count) of the stencil
    inputs of a handle: the five primitives and the temperature (FP64 on the
    plain path, FP32 on the mixed path).  A plane of the padded layout is
    contiguous (sy * px elements), so each field's range is one tensor."""
    import torch
    from . import _lib
    out = []
    for what in (_lib.NS3D_PRIMITIVE, _lib.NS3D_TEMPERATURE):
        ptrs, lay = solver.device_fields(what)
        sx, sy, sz, px, off, esz = lay
        per_plane = sy * px
        start = ((k0 + 3) * per_plane + off) * esz  # ghost-inclusive plane k0 + 3
        ts = "<f8" if esz == 8 else "<f4"
        for p in ptrs:
            if p:
                out.append(torch.as_tensor(_DeviceArray(p + start, count * per_plane, ts), device="cuda"))
    return out


class SlabSolver:
    """One rank's z-slab of a periodic-in-z or bounded domain on one GPU.

    ``exchange_fn(plan, planes)`` moves the halo planes between ranks; the
    default is ``exchange`` over torch.distributed (NCCL on GPUs).  A caller
    that holds every rank's solver in one process can pass its own (device
    copies between the handles)."""

    def __init__(self, P, G, plan: SlabPlan, device: int = 0, exchange_fn=None, allreduce_min=None,
                 allreduce_sum=None, stream=None):
        from .config import BCType, GridDesc
        from .solver import Solver
        import copy
        self.plan = plan
        self.G = G
        Pl = copy.copy(P)
        if plan.world > 1:
            # a halo side is a non-periodic boundary of the local handle;
            # Outflow stands in (its treatment stays inside the halo)
            Pl.bc_zmin = BCType.Outflow if plan.lower is not None else P.bc_zmin
            Pl.bc_zmax = BCType.Outflow if plan.upper is not None else P.bc_zmax
        Gl = copy.copy(G)
        Gl.global_nz = plan.nz_local
        Gl.Lz = G.dz * plan.nz_local
        Gl.dz = G.dz
        self.P, self.Gl = Pl, Gl
        self.s = Solver(Pl, Gl, device=device)
        # the stages and the halo moves must be ordered: the handle and the
        # torch copies / NCCL operations of the exchange run on one explicit
        # (non-default) stream; ns3d_set_stream(NULL) would give the handle a
        # private stream of its own
        import torch
        self.stream = stream if stream is not None else torch.cuda.Stream(device=device)
        self.s.set_stream(self.stream.cuda_stream)
        if plan.world > 1:
            # the global spacing, bit for bit (Lz / nz of the local extent may round differently)
            self.s._check(self.s.lib.ns3d_set_slab(self.s.h, plan.zlo, plan.zhi, float(G.dz), int(plan.periodic)))
        self._exchange = exchange_fn or (lambda pl, planes: exchange(pl, planes))
        self._min = allreduce_min or _dist_allreduce(min_op=True)
        self._sum = allreduce_sum or _dist_allreduce(min_op=False)

    def close(self):
        self.s.close()

    # -- state
    def local_block(self, field: np.ndarray) -> np.ndarray:
        """The local interior planes (owned + halo) of a global interior field (nz, ny, nx)."""
        return field[self.plan.global_planes()]

    def set_interior_primitives(self, rho, u, v, w, p) -> None:
        self.s.set_interior_primitives(*[self.local_block(f) for f in (rho, u, v, w, p)])

    def owned(self, arr: np.ndarray) -> np.ndarray:
        """Owned planes of a downloaded Field3D group (..., sz, sy, sx) (ghost-inclusive)."""
        return arr[..., 3 + self.plan.zlo:3 + self.plan.zhi, :, :]

    def planes(self, side: str, k0: int, count: int):
        return device_planes(self.s, k0, count)

    def exchange_halos(self) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            self._exchange(self.plan, self.planes)

    # -- time advance
    launch_count = 0  # kernels this rank's handle launched (ns3d_last_launch_count summed)

    def compute_timestep(self) -> float:
        import torch
        dt = self.s.compute_timestep()
        self.launch_count += self.s.launches()
        with torch.cuda.stream(self.stream):
            return self._min(dt)

    def total_energy(self) -> float:
        import torch
        ke = self.s.total_energy()
        with torch.cuda.stream(self.stream):
            return self._sum(ke)

    def rk3_step(self, dt: float) -> None:
        for stage in (1, 2, 3):
            self.s._check(self.s.lib.ns3d_rk3_stage(self.s.h, stage, float(dt)))
            self.launch_count += self.s.launches()
            self.exchange_halos()


def _dist_allreduce(min_op: bool):
    def f(x: float) -> float:
        import torch
        import torch.distributed as dist
        if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
            return x
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if min_op else dist.ReduceOp.SUM)
        return float(t.item())
    return f


class InProcessSlabs:
    """Every rank's SlabSolver in one process on one GPU, the halo exchange
    done by device-to-device copies between the handles, all on the current
    stream.  No kernel waits on another rank: the host orders the stage
    launches of all slabs, then the copies.  Used to check the decomposition
    against a single-domain run on one device."""

    def __init__(self, P, G, world: int, device: int = 0):
        import torch
        periodic = P.bc_zmin == P.bc_zmax and int(P.bc_zmin) == 0
        self.plans = [slab_plan(G.global_nz, world, r, periodic) for r in range(world)]
        ident = lambda x: x
        # one stream for every slab's kernels and for the copies between them
        self.stream = torch.cuda.Stream(device=device)
        self.slabs = [SlabSolver(P, G, pl, device=device, exchange_fn=lambda *_: None, allreduce_min=ident,
                                 allreduce_sum=ident, stream=self.stream) for pl in self.plans]

    def close(self):
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_interior_primitives(self, rho, u, v, w, p) -> None:
        for s in self.slabs:
            s.set_interior_primitives(rho, u, v, w, p)

    def exchange_halos(self) -> None:
        import torch
        with torch.cuda.stream(self.stream):
            self._copy_halos()

    def _copy_halos(self) -> None:
        for s in self.slabs:
            pl = s.plan
            if pl.lower is not None:
                src = self.slabs[pl.lower]
                for d, t in zip(s.planes("recv", pl.zlo - HALO, HALO), src.planes("send", src.plan.zhi - HALO, HALO)):
                    d.copy_(t)
            if pl.upper is not None:
                src = self.slabs[pl.upper]
                for d, t in zip(s.planes("recv", pl.zhi, HALO), src.planes("send", src.plan.zlo, HALO)):
                    d.copy_(t)

    def compute_timestep(self) -> float:
        return min(s.s.compute_timestep() for s in self.slabs)

    def total_energy(self) -> float:
        return sum(s.s.total_energy() for s in self.slabs)

    def rk3_step(self, dt: float) -> None:
        for stage in (1, 2, 3):
            for s in self.slabs:
                s.s._check(s.s.lib.ns3d_rk3_stage(s.s.h, stage, float(dt)))
            self.exchange_halos()

    def owned_primitives(self) -> np.ndarray:
        """The owned planes of every slab, stacked along z: (5, nz, sy, sx)."""
        return np.concatenate([s.owned(s.s.primitives()) for s in self.slabs], axis=1)
