"""Hand-written VJPs of the face flux and of the node viscous flux, checked
against central finite differences of the production forward code (host
evaluation through ns3d_debug_*; no device needed)."""
import ctypes as C

import numpy as np
import pytest

from ns3d_wcns_b200 import _lib, build

_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def p(a):
    return a.ctypes.data_as(_dp)


def random_stencil(rng, jump=False):
    g = 1.4
    rho = 1.0 + 0.2 * rng.uniform(-1, 1, 6)
    vel = rng.uniform(-1, 1, (3, 6))
    pr = 7.9 * (1.0 + 0.1 * rng.uniform(-1, 1, 6))
    if jump:
        rho[3:] *= 0.4
        pr[3:] *= 0.3
    U = np.empty((5, 6))
    U[0] = rho
    U[1:4] = rho * vel
    U[4] = pr / (g - 1) + 0.5 * rho * (vel ** 2).sum(0)
    return U


LIN = np.array([0.0248, -0.2015, 0.6952, 0.5734, -0.0848, -0.0071])
# MDCD_HYBRID's WENO weights d0..d3 for mdcd_disp 0.0463783, mdcd_diss 0.01
# (interpolation.cpp:179-182), appended to the linear coefficients
HD = np.array([1.5 * (0.0463783 + 0.01), 0.5 - 1.5 * (0.0463783 - 0.03), 0.5 - 1.5 * (0.0463783 + 0.03),
               1.5 * (0.0463783 - 0.01)])


@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("interp", [0, 2, 3])
@pytest.mark.parametrize("riemann", [0, 1, 2, 3])
def test_face_vjp_matches_finite_differences(lib, direction, interp, riemann):
    """Roe, Rusanov, HLLC (public value 2) and HLL (3) with WENO5,
    MDCD_LINEAR and MDCD_HYBRID (detector switch: zero derivative, active
    branch differentiated)."""
    rng = np.random.default_rng(100 * direction + 10 * interp + riemann)
    lin = np.ascontiguousarray(np.concatenate([LIN, HD]))
    worst, kinks = 0.0, 0

    def fd(U, dU, Fb, h):
        Fp, Fm, tmp = np.zeros(5), np.zeros(5), np.zeros(30)
        lib.ns3d_debug_face_vjp(direction, interp, riemann, 1.4, p(lin),
                                p(np.ascontiguousarray((U + h * dU).ravel())), p(Fb), p(tmp), p(Fp))
        lib.ns3d_debug_face_vjp(direction, interp, riemann, 1.4, p(lin),
                                p(np.ascontiguousarray((U - h * dU).ravel())), p(Fb), p(tmp), p(Fm))
        return Fb @ (Fp - Fm) / (2 * h)

    for trial in range(12):
        U = random_stencil(rng, jump=trial % 3 == 2)
        Fb = rng.standard_normal(5)
        dU = rng.standard_normal((5, 6)) * np.abs(U).mean(axis=1, keepdims=True)
        out = np.zeros(30)
        F = np.zeros(5)
        assert lib.ns3d_debug_face_vjp(direction, interp, riemann, 1.4, p(lin), p(np.ascontiguousarray(U.ravel())),
                                       p(Fb), p(out), p(F)) == 0
        f1, f2 = fd(U, dU, Fb, 1e-6), fd(U, dU, Fb, 1e-7)
        if abs(f1 - f2) > 1e-5 * max(abs(f1), 1e-3):
            kinks += 1  # the finite difference straddles a switch (max/abs/branch): not a derivative
            continue
        ad = out @ dU.ravel()
        worst = max(worst, abs(f1 - ad) / max(abs(f1), 1e-3))
    assert kinks <= 2 and worst < 2e-6, (worst, kinks)


def test_viscous_vjp_matches_finite_differences(lib):
    rng = np.random.default_rng(7)
    mu0, S, cpr = 1.0 / 200, 110.4 / 273.15, 1.0 / (1.4 * 0.4 * 0.09) * 1.4 / 0.72
    for _ in range(10):
        x = np.array([rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.8, 1.2)])
        g = rng.standard_normal(12)
        Vb = rng.standard_normal(9)
        xb, gb, V = np.zeros(4), np.zeros(12), np.zeros(9)
        lib.ns3d_debug_visc_vjp(mu0, S, cpr, p(x), p(g), p(Vb), p(xb), p(gb), p(V))
        dx, dg = rng.standard_normal(4) * 0.1, rng.standard_normal(12)
        h = 1e-6
        Vp, Vm, t4, t12 = np.zeros(9), np.zeros(9), np.zeros(4), np.zeros(12)
        lib.ns3d_debug_visc_vjp(mu0, S, cpr, p(x + h * dx), p(g + h * dg), p(Vb), p(t4), p(t12), p(Vp))
        lib.ns3d_debug_visc_vjp(mu0, S, cpr, p(x - h * dx), p(g - h * dg), p(Vb), p(t4), p(t12), p(Vm))
        fd = Vb @ (Vp - Vm) / (2 * h)
        ad = xb @ dx + gb @ dg
        assert abs(fd - ad) <= 1e-7 * max(abs(fd), 1e-3)
