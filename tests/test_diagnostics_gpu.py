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


def test_fused_diagnostics_equal_separate_pass(gpu_lib, monkeypatch):
    """ns3d_diagnostics (FP64) sums |grad u|^2, mu, rho, |u|^2 and the kinetic
    energy in a pass built from the viscous kernel (its TMA plane tiles and
    register windows, sums instead of node fluxes).  Every output equals the
    separate per-cell gradient pass (NS3D_DIAG_SEPARATE=1) to 1e-13 relative
    -- the same terms summed in another fixed order -- and the trajectory does
    not depend on whether the monitor ran: a step taken after the diagnostics
    equals one taken without them bit for bit."""
    from ns3d_wcns_b200.solver import Solver
    n = (24, 20, 18)
    P, G = make_params(n=n, L=(2 * math.pi, 1.7 * math.pi, 1.5 * math.pi), Ma=0.3, Re=400.0, interpolation=3,
                       riemann=2, cfl=0.5, dt_fixed=-1.0)
    st = isotropic_state(n, 1.4, 0.3, seed=6)
    out = {}
    for mode in ("fused", "separate"):
        if mode == "separate":
            monkeypatch.setenv("NS3D_DIAG_SEPARATE", "1")
        else:
            monkeypatch.delenv("NS3D_DIAG_SEPARATE", raising=False)
        with Solver(P, G) as s:
            s.set_interior_primitives(*st)
            for _ in range(2):
                s.rk3_step(s.compute_timestep())
            d = np.array(list(s.diagnostics().values()))
            s.rk3_step(s.compute_timestep())
            out[mode] = (d, s.primitives())
    monkeypatch.delenv("NS3D_DIAG_SEPARATE", raising=False)
    a, b = out["fused"][0], out["separate"][0]
    assert np.all(np.abs(a - b) <= 1e-13 * np.abs(b)), (a, b)
    assert np.array_equal(out["fused"][1], out["separate"][1])
