"""z-slab decomposition on one GPU: every rank's slab as its own handle in
one process, the halo planes exchanged by device copies between the handles
after every RK stage (the multi-GPU path moves the same planes with NCCL
point-to-point operations).  The owned planes of every slab must equal a
single-domain run bit for bit -- state, time step -- and the kinetic energy
(a sum in another order) to 1e-13.  Cases: periodic z (every slab has two
halos), Wall/Outflow z (the end slabs have a real boundary), both
precisions, two to four slabs of unequal size."""
import math

import numpy as np
import pytest

from helpers import interior
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("world,bcs", [(2, (0,) * 6), (3, (0,) * 6), (4, (0, 0, 0, 0, 1, 3))],
                         ids=["2-periodic", "3-periodic", "4-wall-outflow"])
def test_slabs_equal_single_domain(gpu_lib, precision, world, bcs):
    from ns3d_wcns_b200.slab import InProcessSlabs
    from ns3d_wcns_b200.solver import Solver
    n = (24, 20, 38)
    P, G = make_params(n=n, L=(2 * math.pi, 1.6 * math.pi, 3 * math.pi), Ma=0.3, Re=400.0, cfl=0.5,
                       dt_fixed=-1.0, interpolation=3, riemann=2, bcs=bcs, precision=precision)
    st = random_state(n, seed=3, amp=0.2) if bcs[4] else isotropic_state(n, P.gamma, P.Ma, seed=3)
    with Solver(P, G) as ref, InProcessSlabs(P, G, world) as slabs:
        ref.set_interior_primitives(*st)
        slabs.set_interior_primitives(*st)
        for step in range(4):
            dt = ref.compute_timestep()
            dts = slabs.compute_timestep()
            assert dts == dt, (step, dts, dt)
            ref.rk3_step(dt)
            slabs.rk3_step(dt)
        W = ref.primitives()[:, 3:-3]
        Ws = slabs.owned_primitives()
        # owned interior cells and their x/y ghosts, every variable, bit for bit
        assert np.array_equal(Ws, W), np.abs(Ws - W).max()
        ke, kes = ref.total_energy(), slabs.total_energy()
        assert abs(kes - ke) <= 1e-13 * ke, (kes, ke)


def test_slab_refuses_whole_step_calls(gpu_lib):
    from ns3d_wcns_b200 import _lib
    from ns3d_wcns_b200.slab import InProcessSlabs
    n = (16, 12, 24)
    P, G = make_params(n=n, interpolation=0, riemann=0)
    with InProcessSlabs(P, G, 2) as slabs:
        slabs.set_interior_primitives(*random_state(n, seed=1))
        s = slabs.slabs[0].s
        with pytest.raises(_lib.Ns3dError):
            s.rk3_step(1e-4)
        with pytest.raises(_lib.Ns3dError):
            s.time_advance(1.0, 2)
        # stages must come in order
        assert s.lib.ns3d_rk3_stage(s.h, 2, 1e-4) == -7
