"""GPU parity through the C ABI against the oracle (the reference's algorithm
restated in C and pinned bit-for-bit to the reference) and against the
reference's own golden outputs.

Tolerances (plain FP64 path): relative L-infinity 1e-12 on one RHS, 1e-10
after 10 RK3 steps -- relative to max|reference| per variable.
"""
import os

import numpy as np
import pytest

from helpers import golden_cases, interior, params_from_cfg, rel_linf
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state
from oracle import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = np.load(os.path.join(HERE, "golden", "ref_cases.npz"))
RHS_TOL = 1e-12
STEP_TOL = 1e-10


def solver(P, G):
    from ns3d_wcns_b200.solver import Solver
    return Solver(P, G)


def per_var(a, b):
    return max(rel_linf(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("interp", [0, 2, 3])
@pytest.mark.parametrize("rs", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("ch", [0, 1])
def test_rhs_all_schemes_periodic(gpu_lib, interp, rs, ch):
    n = (9, 7, 6)
    P, G = make_params(n=n, L=(1.0, 0.8, 0.7), interpolation=interp, riemann=rs, char_recon=ch)
    st = random_state(n, seed=5 + rs)
    o = oracle.PortSolver(P, G)
    o.set_interior_prims(*st)
    o.compute_rhs()
    with solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.compute_rhs()
        assert per_var(interior(s.rhs()), interior(o.rhs())) <= RHS_TOL
        # state after the device ghost fill, every cell (ghosts included)
        W = s.primitives()
        ref = np.stack([o.get(k) for k in ("rho", "u", "v", "w", "p")])
        assert np.array_equal(W, ref)


BCS = [(3, 3, 3, 3, 3, 3), (1, 1, 2, 2, 3, 3), (4, 3, 0, 0, 1, 2), (1, 2, 4, 3, 3, 4), (2, 2, 1, 1, 4, 4)]


@pytest.mark.parametrize("bcs", BCS)
@pytest.mark.parametrize("scheme", [(0, 0, 0), (3, 2, 0), (2, 4, 1)])
def test_rhs_and_steps_nonperiodic(gpu_lib, bcs, scheme):
    n = (10, 7, 8)
    interp, rs, ch = scheme
    P, G = make_params(n=n, L=(1.0, 0.9, 1.1), interpolation=interp, riemann=rs, char_recon=ch, bcs=bcs)
    st = random_state(n, seed=3, amp=0.2)
    o = oracle.PortSolver(P, G)
    o.set_interior_prims(*st)
    o.compute_rhs()
    with solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.compute_rhs()
        assert per_var(interior(s.rhs()), interior(o.rhs())) <= RHS_TOL
        for _ in range(3):
            o.rk3_step(2e-4)
            s.rk3_step(2e-4)
        assert per_var(s.conserved(), o.conserved()) <= STEP_TOL


@pytest.mark.parametrize("name,cfg", golden_cases(CASES), ids=[n for n, _ in golden_cases(CASES)])
def test_against_reference_golden(gpu_lib, name, cfg):
    P, G = params_from_cfg(cfg)
    with solver(P, G) as s:
        s.set_interior_primitives(*CASES[name + "_in"])
        s.compute_rhs()
        ref_rhs = CASES[name + "_rhs"]
        got = interior(s.rhs())
        finite = np.isfinite(ref_rhs)
        assert np.array_equal(finite, np.isfinite(got))
        assert max(rel_linf(g[f], r[f]) for g, r, f in zip(got, ref_rhs, finite)) <= RHS_TOL
        for _ in range(cfg["steps"]):
            s.rk3_step(cfg["dt"])
        U, ref_U = s.conserved(), CASES[name + "_U"]
        finite = np.isfinite(ref_U)
        assert np.array_equal(finite, np.isfinite(U))
        assert max(rel_linf(g[f], r[f]) for g, r, f in zip(U, ref_U, finite)) <= STEP_TOL
        if np.isfinite(CASES[name + "_dt"]):
            assert abs(s.compute_timestep() - float(CASES[name + "_dt"])) <= 1e-14 * float(CASES[name + "_dt"])


def test_config1_ten_steps_32cubed(gpu_lib):
    """Isotropic turbulence 32^3, WENO5 + Roe, Ma 0.3, Re 100, dt 1e-3, 10 steps:
    the full conserved field against the oracle."""
    n = (32, 32, 32)
    P, G = make_params(n=n, Ma=0.3, Re=100.0, Pr=0.72, S_ref=110.4 / 273.15)
    st = isotropic_state(n, P.gamma, P.Ma, seed=0)
    o = oracle.PortSolver(P, G)
    o.set_interior_prims(*st)
    o.compute_rhs()
    with solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.compute_rhs()
        assert per_var(interior(s.rhs()), interior(o.rhs())) <= RHS_TOL
        for _ in range(10):
            o.rk3_step(1e-3)
        s.rk3_steps(10, 1e-3)
        assert per_var(s.conserved(), o.conserved()) <= STEP_TOL
        assert abs(s.total_energy() - o.total_energy()) <= 1e-13 * o.total_energy()
        assert s.compute_timestep() == o.timestep()


def test_time_advance_adaptive_matches_reference_schedule(gpu_lib):
    """maincycle.cpp's dt schedule with compute_timestep (adaptive) and the last
    step clipped to TotalTime."""
    n = (12, 10, 8)
    P, G = make_params(n=n, L=(2 * np.pi,) * 3, Ma=0.3, Re=400.0, cfl=0.5, dt_fixed=-1.0, interpolation=3,
                       riemann=2)
    st = isotropic_state(n, P.gamma, P.Ma, seed=2)
    o = oracle.PortSolver(P, G)
    o.set_interior_prims(*st)
    t_end = 0.05
    t, steps = 0.0, 0
    while abs(t_end - t) > 1e-12 and steps < 100:
        dt = o.timestep()
        if t + dt > t_end:
            dt = t_end - t
        t += dt
        o.rk3_step(dt)
        steps += 1
        if t >= t_end:
            break
    with solver(P, G) as s:
        s.set_interior_primitives(*st)
        tg, ng = s.time_advance(t_end, 100)
        assert ng == steps and tg == t
        assert per_var(s.conserved(), o.conserved()) <= STEP_TOL


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("bcs", [(0,) * 6, (3, 3, 1, 2, 0, 0)])
def test_cfl_fused_into_last_stage(gpu_lib, precision, bcs):
    """The time step right after an RK3 step comes from the per-block minima
    written by the last stage; it equals the separate reduction's bit for bit.
    The kinetic energy of the new state comes from the same stage's block sums."""
    n = (20, 14, 12)
    P, G = make_params(n=n, L=(1.0, 0.7, 0.6), interpolation=3, riemann=2, bcs=bcs, cfl=0.5, dt_fixed=-1.0,
                       Re=300.0, precision=precision)
    with solver(P, G) as s:
        s.set_interior_primitives(*random_state(n, seed=5))
        for _ in range(3):
            dt = s.compute_timestep()
            s.rk3_step(dt)
            fused = s.compute_timestep()
            ke_fused = s.total_energy()
            s.apply_boundary()  # unchanged state, forces the separate reductions
            plain = s.compute_timestep()
            assert fused == plain, (fused, plain)
            # kinetic energy: the same sum in another (fixed) order
            ke_plain = s.total_energy()
            assert abs(ke_fused - ke_plain) <= 1e-13 * abs(ke_plain), (ke_fused, ke_plain)


@pytest.mark.parametrize("precision", [0, 1])
def test_rhs_after_step_kept_on_request(gpu_lib, precision):
    """runge_kutta_3 leaves its last stage's right-hand side in F.rhs_*
    (range_kutta.cpp:80-88).  With keep_rhs the fused last stage stores it
    too; without it the RHS buffer holds a partial sum after a step, and its
    download is refused rather than handing that back.  FP64: relative
    L-infinity 1e-12 against the oracle; mixed (continuous MDCD_LINEAR, so
    no detector flips): relative L2 1e-4 per variable."""
    from ns3d_wcns_b200 import _lib
    from ns3d_wcns_b200 import analysis
    from ns3d_wcns_b200.solver import Solver
    n = (12, 10, 8)
    interp = 3 if precision == 0 else 2
    kw = dict(n=n, L=(1.0, 0.8, 0.7), interpolation=interp, riemann=2, bcs=(3, 3, 0, 0, 1, 2))
    P, G = make_params(precision=precision, **kw)
    st = random_state(n, seed=6, amp=0.2)
    o = oracle.PortSolver(make_params(**kw)[0], G)
    o.set_interior_prims(*st)
    for _ in range(2):
        o.rk3_step(3e-4)
    with Solver(P, G, keep_rhs=True) as s:
        s.set_interior_primitives(*st)
        s.rk3_steps(2, 3e-4)
        got, ref = interior(s.rhs()), interior(o.rhs())
        if precision == 0:
            err = per_var(got, ref)
            assert err <= RHS_TOL, err
        else:
            err = max(analysis.rel_l2(a, b) for a, b in zip(got, ref))
            assert err <= 1e-4, err
        # the device time loop keeps it as well
        t, k = s.time_advance(1.0, 1)
        assert k == 1
        s.rhs()
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.rk3_step(3e-4)
        with pytest.raises(_lib.Ns3dError) as e:
            s.rhs()
        assert e.value.status == -7
        s.compute_rhs()
        s.rhs()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")
@pytest.mark.parametrize("kind", ["riemann_2d", "sod", "uniform", "sine_x"])
@pytest.mark.parametrize("bcs", [(0,) * 6, (3, 3, 1, 2, 0, 0)])
def test_device_initialisers(gpu_lib, kind, bcs):
    """The reference's built-in initialisers run on the device, then the ghost
    fill, against the reference's own initialise + apply_boundary +
    primitiveToConserved (main.cpp:85-99): every cell, ghosts included.
    Bit for bit, except sine_x, whose sin() may differ in the last bit between
    CUDA and the host C library (relative 1e-15)."""
    n = (12, 10, 6)
    P, G = make_params(n=n, L=(1.0, 1.0, 0.5), bcs=bcs)
    ref = oracle.RefSolver(P, G)
    ref.initialize(kind)
    with solver(P, G) as s:
        s.initialize(kind)
        W = s.primitives()
        U = s.conserved()
    Wr = np.stack([ref.get(k) for k in ("rho", "u", "v", "w", "p")])
    Ur = ref.conserved()
    if kind == "sine_x":
        assert per_var(W, Wr) <= 1e-15 and per_var(U, Ur) <= 1e-15
    else:
        assert np.array_equal(W, Wr) and np.array_equal(U, Ur)
    # and the state then steps like the reference's (relative to the largest
    # conserved value: w, and v for sod / sine_x, stay zero up to rounding)
    ref.rk3_step(1e-4)
    with solver(P, G) as s:
        s.initialize(kind)
        s.rk3_step(1e-4)
        U, Ur = s.conserved(), ref.conserved()
        assert np.abs(U - Ur).max() <= STEP_TOL * np.abs(Ur).max()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")
@pytest.mark.parametrize("n", [(8, 6, 4), (16, 12, 10), (24, 20, 18)])
def test_device_isotropic_initialiser(gpu_lib, n):
    """init_isotropic_turbulence (isotropic_ini.cpp:131-193) on the device: the
    seed-123 std::mt19937_64 phases, the k0 = 8 spectrum, its inverse transform
    (a direct DFT here, FFTW in the reference: the same sums in another order)
    and the energy normalisation, then the ghost fill -- against the
    reference's own initialiser + apply_boundary + primitiveToConserved, every
    cell: rho and p exactly, the velocity to 1e-12 of its largest value.  A
    second call starts from the seed again."""
    P, G = make_params(n=n)
    ref = oracle.RefSolver(P, G)
    ref.initialize("isotropic")
    Wr = np.stack([ref.get(k) for k in ("rho", "u", "v", "w", "p")])
    with solver(P, G) as s:
        s.initialize("isotropic")
        W = s.primitives()
        s.initialize("isotropic")
        assert np.array_equal(s.primitives(), W)
    assert np.array_equal(W[0], Wr[0]) and np.array_equal(W[4], Wr[4])
    err = np.abs(W[1:4] - Wr[1:4]).max() / np.abs(Wr[1:4]).max()
    print("isotropic initialiser, velocity error relative to its largest value:", err)
    assert err <= 1e-12
