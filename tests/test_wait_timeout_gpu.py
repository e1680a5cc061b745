"""Failure path of the device-side waits: a bounded mbarrier wait that runs out
writes the device error word and returns; the host reports NS3D_ERR_TIMEOUT and
the device stays usable (a solver step runs right after)."""
import ctypes as C

import pytest

from ns3d_wcns_b200 import _lib
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import random_state

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_reports(gpu_lib):
    code = C.c_int(0)
    r = gpu_lib.ns3d_debug_wait_timeout(0, 1 << 12, C.byref(code))
    assert r == -9 and code.value == 1, (r, code.value)  # NS3D_ERR_TIMEOUT, the TMA-timeout code
    # the context is intact: the solver (whose viscous kernel waits on TMA tiles) still runs
    from ns3d_wcns_b200.solver import Solver
    n = (12, 10, 9)
    P, G = make_params(n=n, interpolation=3, riemann=2, Re=200.0)
    with Solver(P, G) as s:
        s.set_interior_primitives(*random_state(n, seed=1))
        s.rk3_step(1e-4)
        assert s.total_energy() > 0
