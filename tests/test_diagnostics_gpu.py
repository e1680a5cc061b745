"""On-GPU turbulence statistics (Solver.turbulence_stats: zero-copy views of the
resident fields, FFT spectrum and dissipation on the device) against the same
statistics of the downloaded host arrays, and the kinetic energy against the
library's own reduction."""
import math

import numpy as np
import pytest

from helpers import interior
from ns3d_wcns_b200 import analysis
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_device_stats_match_host_stats(gpu_lib, precision):
    from ns3d_wcns_b200.solver import Solver
    n = 32
    P, G = make_params(n=(n, n, n), L=(2 * math.pi,) * 3, Ma=0.3, Re=400.0, interpolation=3, riemann=2,
                       S_ref=110.4 / 273.15, precision=precision)
    with Solver(P, G) as s:
        s.set_interior_primitives(*isotropic_state((n, n, n), 1.4, 0.3, seed=2))
        s.rk3_step(s.compute_timestep())
        dev = s.turbulence_stats()
        W = interior(s.primitives())
        T = interior(s.temperature())
        ke_lib = s.total_energy()
    host = analysis.turbulence_stats(W[0], W[1], W[2], W[3], T, 1.0 / 400.0, 110.4 / 273.15,
                                     (2 * math.pi / n) ** 3)
    for k in ("total_energy", "kinetic_energy", "u_rms", "mean_mu", "mean_rho", "dissipation"):
        assert abs(dev[k] - host[k]) <= 1e-12 * abs(host[k]), (k, dev[k], host[k])
    np.testing.assert_allclose(dev["spectrum"], host["spectrum"], rtol=1e-10, atol=1e-14)
    assert abs(dev["total_energy"] - ke_lib) <= 1e-12 * ke_lib
