"""time_advance with its dt schedule on the device (steps captured in CUDA
graphs, one host synchronisation per graph launch) against the host loop of
the same entry point (taken when per-kernel profiling is on): the same step
count, time and state, bit for bit."""
import math

import numpy as np
import pytest

from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state

pytestmark = pytest.mark.gpu


def _run(P, G, st, t_end, max_steps, host_loop, t0=0.0):
    from ns3d_wcns_b200.solver import Solver
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        if host_loop:
            s.profile(True)
        t, n = s.time_advance(t_end, max_steps, t0)
        t2, n2 = s.time_advance(t_end + 0.01, 5, t)  # a second call continues from there
        return t, n, t2, n2, s.primitives(), s.compute_timestep()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", ["adaptive", "budget", "fixed", "walls"])
def test_device_time_loop_equals_host_loop(gpu_lib, precision, case):
    n = (24, 20, 16)
    bcs = (3, 3, 1, 2, 0, 0) if case == "walls" else (0,) * 6
    P, G = make_params(n=n, L=(2 * math.pi,) * 3, Ma=0.3, Re=400.0, interpolation=3, riemann=2, cfl=0.5,
                       dt_fixed=(2e-3 if case == "fixed" else -1.0), bcs=bcs, precision=precision)
    st = random_state(n, seed=4) if case == "walls" else isotropic_state(n, 1.4, 0.3, seed=6)
    t_end, max_steps = (0.6, 7) if case == "budget" else (0.6, 100000)
    dev = _run(P, G, st, t_end, max_steps, host_loop=False)
    host = _run(P, G, st, t_end, max_steps, host_loop=True)
    assert dev[0] == host[0] and dev[1] == host[1], (dev[:2], host[:2])
    assert dev[2] == host[2] and dev[3] == host[3], (dev[2:4], host[2:4])
    if case == "budget":
        assert dev[1] == 7
    else:
        assert abs(dev[0] - t_end) < 1e-12 and dev[1] > 12  # more than one graph launch
    np.testing.assert_array_equal(dev[4], host[4])
    assert dev[5] == host[5]
