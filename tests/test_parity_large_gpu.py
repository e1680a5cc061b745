"""Field-by-field parity at the benchmark's schemes and at grids that fill
several blocks, bundles and chunks in every direction, against the reference
compiled in place (oracle/_ref, ``oracle.RefSolver``) where it is built, else
against the C restatement (``oracle.PortSolver``, pinned bit for bit to it).

The small-grid parity tests cover every scheme combination; these cover the
instantiations and tilings the 256^3 benchmark runs:
  * 64^3 isotropic turbulence, MDCD_HYBRID + HLLC, Re 400, CFL 0.5 adaptive
    (the oracle-sized case of the benchmark workload), also MDCD_LINEAR +
    HLLC and WENO5 + Roe with characteristic reconstruction;
  * a non-cubic all-periodic 70 x 66 x 40 grid: three x-chunks per line,
    three y/z bundles (the last partial), nine y-chunks and six z-chunks,
    two z-segments of the viscous kernel.
Tolerances (relative L-infinity over every cell, ghosts included, per
variable): 1e-12 for one RHS, 1e-10 after 10 RK3 steps.  The solenoidal
isotropic field makes the continuity and energy right-hand sides small
against the fluxes they are differences of (max |RHS_rho| = 0.2 at 64^3
against momentum fluxes of ~10), so their rounding floor lies above 1e-12:
perturbing the oracle's own inputs by +-1 ulp moves RHS_rho by ~3e-11 of
its maximum.  Each variable's RHS bound is therefore max(1e-12, 4 x that
measured 1-ulp sensitivity), computed in the test.  The time step of
each step is the oracle's; the GPU's own compute_timestep must agree with
it bit for bit at step 0 (identical state) and to 1e-13 relative after that
(the states then differ by rounding: the RHS sums in another order).

The MDCD_HYBRID detector is the one discontinuous decision of the scheme.
The device takes the reference's decision exactly (a cross-multiplied test
far from the threshold, the reference's quotient near it); the planted
near-threshold stencils below check that decision against the quotient.
"""
import math

import numpy as np
import pytest

from helpers import interior, rel_linf
from ns3d_wcns_b200 import analysis
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state
from oracle import oracle

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
STEP_TOL = 1e-10
DT_TOL = 1e-13
MDCD_EPS = 0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4


def _oracle(P, G):
    return oracle.RefSolver(P, G) if oracle.ref_available() else oracle.PortSolver(P, G)


def _per_var(a, b):
    return max(rel_linf(x, y) for x, y in zip(a, b))


def _sai_quotient(a, b):
    """The reference's detector value (interpolation.cpp:157-158): numpy
    float64 operations are unfused IEEE, as in the reference build."""
    return (2 * a * b + MDCD_EPS) / (a * a + b * b + MDCD_EPS)


def _sai_cross(a, b):
    """The cross-multiplied comparison without the near-threshold guard."""
    return (2 * a * b + MDCD_EPS) > 0.4 * (a * a + b * b + MDCD_EPS)


def _detector_ab(U, axis):
    """a, b of mdcd_hybrid_interpolate at every cell that has two neighbours
    on each side along `axis` (U: conserved [5, sz, sy, sx])."""
    n = U.shape[axis + 1]

    def sl(o):
        return (slice(None),) + tuple(slice(2 + o, n - 2 + o) if d == axis else slice(None) for d in range(3))

    f = [U[sl(o)] for o in (-2, -1, 0, 1, 2)]
    a = np.abs(f[2] - f[1]) + np.abs(f[2] - 2 * f[1] + f[0])
    b = np.abs(f[2] - f[3]) + np.abs(f[2] - 2 * f[3] + f[4])
    return a, b


def _detector_flips(U):
    """Cells (per variable and direction) where the unguarded cross-multiplied
    test and the reference's quotient decide differently, and cells within
    1e-12 of the threshold (decided by the quotient on the device)."""
    flips = near = 0
    for ax in (2, 1, 0):  # x, y, z in [sz, sy, sx] storage
        a, b = _detector_ab(U, ax)
        q = _sai_quotient(a, b) > 0.4
        flips += int(np.count_nonzero(q != _sai_cross(a, b)))
        lhs, rhs = 2 * a * b + MDCD_EPS, 0.4 * (a * a + b * b + MDCD_EPS)
        near += int(np.count_nonzero(np.abs(lhs - rhs) <= 1e-12 * rhs))
    return flips, near


def _run_pair(P, G, st, steps, count_detector=False):
    from ns3d_wcns_b200.solver import Solver
    o = _oracle(P, G)
    # the rounding floor of each RHS variable: its change under +-1-ulp input perturbations
    rng = np.random.default_rng(0)
    o.set_interior_prims(*[f * (1 + rng.choice([-1.0, 0.0, 1.0], f.shape) * np.finfo(float).eps) for f in st])
    o.compute_rhs()
    R_pert = interior(o.rhs()).copy()
    o.set_interior_prims(*st)
    o.compute_rhs()
    R_ref = interior(o.rhs()).copy()
    sens = [rel_linf(a, b) for a, b in zip(R_pert, R_ref)]
    flips = near = 0
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        s.compute_rhs()
        errs = [rel_linf(a, b) for a, b in zip(interior(s.rhs()), R_ref)]
        rhs_err = max(errs)
        for q in range(5):
            assert errs[q] <= max(RHS_TOL, 4 * sens[q]), (q, errs, sens)
        dt_exact = 0
        for it in range(steps):
            if count_detector:
                f, nr = _detector_flips(o.conserved())
                flips, near = flips + f, near + nr
            if P.dt_fixed > 0:
                dt = P.dt_fixed
            else:
                dt = o.timestep()
                dts = s.compute_timestep()
                if it == 0:
                    assert dts == dt, (dts, dt)
                assert abs(dts - dt) <= DT_TOL * dt, (it, dts, dt)
                dt_exact += int(dts == dt)
            o.rk3_step(dt)
            s.rk3_step(dt)
        step_err = _per_var(s.conserved(), o.conserved())
        prim_err = _per_var(s.primitives(), np.stack([o.get(k) for k in ("rho", "u", "v", "w", "p")]))
        ke_s, ke_o = s.total_energy(), o.total_energy()
    print(f"{G.global_nx}x{G.global_ny}x{G.global_nz} interp {P.interpolation} riemann {P.riemann_solver} "
          f"char {P.char_recon}: rhs {[f'{e:.1e}' for e in errs]} (1-ulp floor {[f'{e:.1e}' for e in sens]}), "
          f"{steps} steps {step_err:.2e} (prims {prim_err:.2e}), "
          f"dt bit-equal {dt_exact}/{steps}, detector flips {flips} near {near}")
    assert step_err <= STEP_TOL, step_err
    assert prim_err <= STEP_TOL, prim_err
    assert abs(ke_s - ke_o) <= 1e-12 * ke_o, (ke_s, ke_o)
    return flips, near


def _iso_params(n, interp, rs, char=0, Re=400.0, precision=0):
    return make_params(n=n, L=(2 * math.pi,) * 3, Ma=0.3, Re=Re, Pr=0.72, cfl=0.5, dt_fixed=-1.0,
                       interpolation=interp, riemann=rs, char_recon=char, S_ref=110.4 / 273.15,
                       precision=precision)


def test_benchmark_scheme_64cubed(gpu_lib):
    """The benchmark workload's oracle size: 64^3, MDCD_HYBRID + HLLC, Re 400,
    CFL 0.5 adaptive; one RHS, then 10 steps on the oracle's dt schedule."""
    n = (64, 64, 64)
    P, G = _iso_params(n, 3, 2)
    st = isotropic_state(n, P.gamma, P.Ma, seed=1)
    _run_pair(P, G, st, 10, count_detector=True)


@pytest.mark.parametrize("interp,rs,char", [(2, 2, 0), (0, 0, 1)], ids=["mdcd_linear_hllc", "weno5_roe_char"])
def test_other_schemes_64cubed(gpu_lib, interp, rs, char):
    n = (64, 64, 64)
    P, G = _iso_params(n, interp, rs, char)
    st = isotropic_state(n, P.gamma, P.Ma, seed=2)
    _run_pair(P, G, st, 10)


def test_noncubic_multi_tile_periodic(gpu_lib):
    """70 x 66 x 40 all-periodic: every sweep runs several chunks and bundles
    per block row (the last bundle partial) and the compile-time periodic
    viscous kernel marches two z-segments."""
    n = (70, 66, 40)
    P, G = _iso_params(n, 3, 2)
    st = isotropic_state(n, P.gamma, P.Ma, seed=4)
    _run_pair(P, G, st, 10)


def _planted_stencils(rng, m):
    """Five-point stencils (-2x, -x, 0, y, 2y), which give a = x, b = y exactly,
    with y/x within a few ulp of the two roots of sai(a, b) = 0.4."""
    x = 10.0 ** rng.uniform(-4, 1, m)
    # 2ab + e = 0.4 (a^2 + b^2 + e), solved for b at given a
    e = MDCD_EPS
    disc = np.sqrt(4 * x * x - 4 * 0.4 * (0.4 * x * x + 0.4 * e - e))
    roots = np.where(rng.integers(0, 2, m) == 0, (2 * x - disc) / 0.8, (2 * x + disc) / 0.8)
    ulps = rng.integers(-6, 7, m)
    y = roots * (1.0 + ulps * np.finfo(np.float64).eps)
    y = np.where(y > 0, y, np.abs(roots))
    s = np.stack([-2 * x, -x, np.zeros(m), y, 2 * y], axis=1)
    a = np.abs(s[:, 2] - s[:, 1]) + np.abs(s[:, 2] - 2 * s[:, 1] + s[:, 0])
    b = np.abs(s[:, 2] - s[:, 3]) + np.abs(s[:, 2] - 2 * s[:, 3] + s[:, 4])
    return s, a, b


def test_detector_decisions_near_threshold(gpu_lib):
    """Near-threshold stencils: the device detector equals the reference's
    quotient decision on every one, including the cases where the unguarded
    cross-multiplied test decides the other way."""
    import ctypes as C
    rng = np.random.default_rng(11)
    s, a, b = _planted_stencils(rng, 200_000)
    # a random smooth/rough background as well
    bg = rng.standard_normal((50_000, 5)) * 10.0 ** rng.uniform(-3, 1, (50_000, 1))
    ab = np.abs(bg[:, 2] - bg[:, 1]) + np.abs(bg[:, 2] - 2 * bg[:, 1] + bg[:, 0])
    bb = np.abs(bg[:, 2] - bg[:, 3]) + np.abs(bg[:, 2] - 2 * bg[:, 3] + bg[:, 4])
    s = np.ascontiguousarray(np.concatenate([s, bg]))
    a, b = np.concatenate([a, ab]), np.concatenate([b, bb])
    ref = (_sai_quotient(a, b) > 0.4).astype(np.int32)
    cross = _sai_cross(a, b).astype(np.int32)
    out = np.empty(len(s), np.int32)
    r = gpu_lib.ns3d_debug_mdcd_detector(0, len(s), s.ctypes.data_as(C.POINTER(C.c_double)),
                                         out.ctypes.data_as(C.POINTER(C.c_int)))
    assert r == 0
    unguarded_flips = int(np.count_nonzero(cross != ref))
    print(f"planted: {len(s)} stencils, unguarded cross-multiplied flips {unguarded_flips}, "
          f"device mismatches {int(np.count_nonzero(out != ref))}")
    assert unguarded_flips > 0  # the planted set does reach the rounding band
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("interp,rs", [(2, 2), (3, 2)], ids=["mdcd_linear_hllc", "mdcd_hybrid_hllc"])
def test_mixed_64cubed_against_fp64(gpu_lib, interp, rs):
    """Mixed path at 64^3 over 10 steps on the FP64 path's dt schedule.
    Continuous scheme (MDCD_LINEAR): relative L2 <= 1e-6 per conserved
    variable.  MDCD_HYBRID: at most 10x the FP64 path's own divergence when
    its initial state is rounded to FP32 (the bound of the 32^3 tests).
    Kinetic energy within 1e-6 relative in both."""
    from ns3d_wcns_b200.solver import Solver
    n = (64, 64, 64)
    st0 = isotropic_state(n, 1.4, 0.3, seed=5)
    st32 = [np.asarray(f, np.float32).astype(np.float64) for f in st0]

    def run(prec, st, dts=None):
        P, G = _iso_params(n, interp, rs, precision=prec)
        out = []
        with Solver(P, G) as s:
            s.set_interior_primitives(*st)
            for it in range(10):
                dt = s.compute_timestep() if dts is None else dts[it]
                out.append(dt)
                s.rk3_step(dt)
            return interior(s.conserved()), s.total_energy(), out

    U64, ke64, dts = run(0, st0)
    Um, kem, _ = run(1, st0, dts)
    mixed = max(analysis.rel_l2(x, y) for x, y in zip(Um, U64))
    assert abs(kem / ke64 - 1) < 1e-6, (kem, ke64)
    if interp == 2:
        print(f"mixed vs fp64 64^3 MDCD_LINEAR: {mixed:.3e}")
        assert mixed <= 1e-6, mixed
    else:
        Up, _, _ = run(0, st32, dts)
        pert = max(analysis.rel_l2(x, y) for x, y in zip(Up, U64))
        print(f"mixed vs fp64 64^3 MDCD_HYBRID: {mixed:.3e}, fp64 under fp32-rounded input {pert:.3e}")
        assert mixed <= 10.0 * pert, (mixed, pert)
