"""z-slab decomposition on the CPU: world_size 2 and 3 gloo ranks (spawned
processes, rendezvous on 127.0.0.1).  Each rank holds only its owned planes
of a periodic isotropic field, receives its six-plane halos through
ns3d_wcns_b200.slab.exchange (torch.distributed point-to-point, the code the
GPU ranks run over NCCL), and computes the right-hand side of its slab with
the CPU oracle, its z boundaries being the halos (any non-periodic type).
The owned planes of every rank's RHS must equal the single-domain oracle's
bit for bit, and the received halos the global field's wrapped planes."""
import copy
import datetime
import os
import socket

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, nz):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from ns3d_wcns_b200.config import BCType, make_params
    from ns3d_wcns_b200.initial import isotropic_state
    from ns3d_wcns_b200.slab import HALO, exchange, slab_plan
    from oracle import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        n = (16, 12, nz)
        # dz = 1/8: the local extents (nz_local / 8) are exact, so every slab's dz is the global one
        P, G = make_params(n=n, L=(2 * np.pi, 1.5 * np.pi, nz / 8.0), Ma=0.3, Re=300.0, interpolation=3,
                           riemann=2)
        st = isotropic_state((16, 12, nz), P.gamma, P.Ma, seed=11)
        plan = slab_plan(nz, world, rank, periodic=True)
        loc = [np.full((plan.nz_local, 12, 16), np.nan) for _ in range(5)]
        for q in range(5):
            loc[q][plan.zlo:plan.zhi] = st[q][plan.z0:plan.z1]
        tens = [torch.from_numpy(a) for a in loc]
        exchange(plan, lambda side, k0, count: [t[k0:k0 + count] for t in tens])
        gp = plan.global_planes()
        for q in range(5):
            assert np.array_equal(loc[q], st[q][gp]), "halo planes differ from the global field"
        Pl = copy.copy(P)
        Pl.bc_zmin = Pl.bc_zmax = BCType.Outflow
        Gl = copy.copy(G)
        Gl.global_nz = plan.nz_local
        Gl.Lz = plan.nz_local / 8.0
        o = oracle.PortSolver(Pl, Gl)
        o.set_interior_prims(*loc)
        o.compute_rhs()
        rhs_loc = o.rhs()[:, 3 + plan.zlo:3 + plan.zhi, 3:-3, 3:-3].copy()
        g = oracle.PortSolver(P, G)
        g.set_interior_prims(*st)
        g.compute_rhs()
        rhs_glob = g.rhs()[:, 3 + plan.z0:3 + plan.z1, 3:-3, 3:-3]
        assert np.array_equal(rhs_loc, rhs_glob), f"rank {rank}: max diff {np.abs(rhs_loc - rhs_glob).max()}"
        assert HALO == 6
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nz", [(2, 20), (3, 22)])
def test_slab_rhs_equals_single_domain_over_gloo(world, nz):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), nz), nprocs=world, join=True)


def test_slab_plan_covers_the_domain():
    from ns3d_wcns_b200.slab import slab_plan
    for nz, world, periodic in [(64, 4, True), (37, 3, False), (256, 8, True), (12, 2, False)]:
        plans = [slab_plan(nz, world, r, periodic) for r in range(world)]
        owned = np.concatenate([np.arange(p.z0, p.z1) for p in plans])
        assert np.array_equal(owned, np.arange(nz))
        for p in plans:
            assert p.owned >= 6 and p.zhi - p.zlo == p.owned
            if p.lower is not None:
                assert plans[p.lower].z1 % nz == p.z0
            if p.upper is not None:
                assert plans[p.upper].z0 == p.z1 % nz
        if not periodic:
            assert plans[0].lower is None and plans[-1].upper is None
    with pytest.raises(ValueError):
        slab_plan(40, 8, 0, True)  # five planes a rank: fewer than the halo
