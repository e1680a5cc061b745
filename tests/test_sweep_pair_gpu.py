"""Mixed path: the two-lines-per-thread FP32 sweep (paired f32x2 arithmetic)
against the one-line-per-thread FP32 sweep it replaces.

Both kernels evaluate the same formulas in FP32; they differ only in where
multiply-adds are fused, so with the continuous schemes (WENO5, MDCD_LINEAR)
one RHS agrees to FP32 rounding: relative L2 <= 2e-6 per variable.  The
MDCD_HYBRID detector switches discontinuously at a threshold, so a face whose
detector value sits at the threshold may take the other branch: for it the
bound is relative L2 <= 1e-4 with at most 0.1 % of the cells off by more
than 1e-5 relative to max|RHS|.  After ten fused RK3 steps the kinetic
energy agrees to 1e-6.
"""
import math

import numpy as np
import pytest

from helpers import interior
from ns3d_wcns_b200 import analysis
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state

pytestmark = pytest.mark.gpu

CONT_TOL = 2e-6
HYB_L2_TOL = 1e-4
HYB_FRAC = 1e-3


def _rhs(P, G, st, scalar, monkeypatch):
    from ns3d_wcns_b200.solver import Solver
    if scalar:
        monkeypatch.setenv("NS3D_SWEEP32", "scalar")
    else:
        monkeypatch.delenv("NS3D_SWEEP32", raising=False)
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.compute_rhs()
        return interior(s.rhs())


@pytest.mark.parametrize("interp,rs", [(3, 2), (2, 2), (0, 0), (0, 1), (2, 5), (3, 6)])
@pytest.mark.parametrize("bcs", [(0,) * 6, (3, 3, 1, 2, 4, 4), (1, 2, 0, 0, 3, 3)])
def test_pair_vs_scalar_rhs(gpu_lib, monkeypatch, interp, rs, bcs):
    n = (24, 18, 20)
    P, G = make_params(n=n, L=(1.0, 0.8, 0.9), interpolation=interp, riemann=rs, bcs=bcs, Re=300.0,
                       precision=1)
    st = random_state(n, seed=11)
    a = _rhs(P, G, st, False, monkeypatch)
    b = _rhs(P, G, st, True, monkeypatch)
    for q in range(5):
        err = analysis.rel_l2(a[q], b[q])
        if interp == 3:
            off = np.abs(a[q] - b[q]) > 1e-5 * np.abs(b[q]).max()
            assert err <= HYB_L2_TOL and off.mean() <= HYB_FRAC, (q, err, off.mean())
        else:
            assert err <= CONT_TOL, (q, err)


def test_pair_fallback_odd_lines(gpu_lib, monkeypatch):
    """Odd line counts across a bundle (nx odd: y and z sweeps) take the
    scalar kernel; the x sweep (ny even) still runs paired."""
    n = (15, 16, 14)
    P, G = make_params(n=n, L=(1.0, 1.0, 1.0), interpolation=2, riemann=2, Re=300.0, precision=1)
    st = random_state(n, seed=3)
    a = _rhs(P, G, st, False, monkeypatch)
    b = _rhs(P, G, st, True, monkeypatch)
    for q in range(5):
        assert analysis.rel_l2(a[q], b[q]) <= CONT_TOL


def test_pair_vs_scalar_fused_steps(gpu_lib, monkeypatch):
    """Ten RK3 steps with the stage fused into the paired z-sweep against the
    scalar kernels' ten steps: same state to 1e-5, kinetic energy to 1e-6."""
    from ns3d_wcns_b200.solver import Solver
    n = 32
    st = isotropic_state((n, n, n), 1.4, 0.3, seed=2)
    P, G = make_params(n=(n, n, n), L=(2 * math.pi,) * 3, Ma=0.3, Re=400.0, cfl=0.5, dt_fixed=-1.0,
                       interpolation=2, riemann=2, precision=1)
    out = {}
    for scalar in (False, True):
        if scalar:
            monkeypatch.setenv("NS3D_SWEEP32", "scalar")
        else:
            monkeypatch.delenv("NS3D_SWEEP32", raising=False)
        with Solver(P, G) as s:
            s.set_interior_primitives(*st)
            for _ in range(10):
                s.rk3_step(s.compute_timestep())
            out[scalar] = (interior(s.conserved()), s.total_energy())
    for q in range(5):
        assert analysis.rel_l2(out[False][0][q], out[True][0][q]) <= 1e-5, q
    assert abs(out[False][1] / out[True][1] - 1) <= 1e-6


def test_pair_narrow_copies(gpu_lib, monkeypatch):
    """nx even but not a multiple of 4: the z sweep stays paired with 8-byte
    copies per pair (its 16-byte copies need four aligned lines)."""
    n = (18, 20, 16)
    P, G = make_params(n=n, L=(1.0, 1.0, 1.0), interpolation=2, riemann=2, Re=300.0, precision=1)
    st = random_state(n, seed=4)
    a = _rhs(P, G, st, False, monkeypatch)
    b = _rhs(P, G, st, True, monkeypatch)
    for q in range(5):
        assert analysis.rel_l2(a[q], b[q]) <= CONT_TOL


@pytest.mark.parametrize("bcs", [(3, 3, 1, 2, 4, 4), (1, 1, 0, 0, 3, 3)])
def test_pair_fused_steps_nonperiodic(gpu_lib, monkeypatch, bcs):
    """Fused RK3 steps (increment form, 16-byte z copies: nx a multiple of 4)
    with non-periodic boundaries in z: paired against scalar kernels to 1e-5,
    and the mixed state against the plain FP64 path to 1e-4 (continuous scheme)."""
    from ns3d_wcns_b200.solver import Solver
    n = (24, 18, 20)
    st = random_state(n, seed=6)
    out = {}
    for key, prec, scalar in (("pair", 1, False), ("scalar", 1, True), ("fp64", 0, False)):
        if scalar:
            monkeypatch.setenv("NS3D_SWEEP32", "scalar")
        else:
            monkeypatch.delenv("NS3D_SWEEP32", raising=False)
        P, G = make_params(n=n, L=(1.0, 0.8, 0.9), interpolation=2, riemann=2, bcs=bcs, Re=300.0,
                           precision=prec, cfl=0.4, dt_fixed=-1.0)
        with Solver(P, G) as s:
            s.set_interior_primitives(*st)
            for _ in range(5):
                s.rk3_step(s.compute_timestep())
            out[key] = interior(s.conserved())
    for q in range(5):
        assert analysis.rel_l2(out["pair"][q], out["scalar"][q]) <= 1e-5, q
        assert analysis.rel_l2(out["pair"][q], out["fp64"][q]) <= 1e-4, q
