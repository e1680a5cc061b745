"""The production face-flux functions (schemes.cuh), evaluated on the host
through ns3d_debug_riemann: consistency F(U, U) = F(U) for every solver, the
Steger-Warming splitting against an independent restatement of the published
formula, and agreement of the six reference solvers with the oracle's known
answers."""
import ctypes as C

import numpy as np
import pytest

from ns3d_wcns_b200 import _lib, build

GAMMA = 1.4
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def flux(lib, d, rs, UL, UR):
    F = np.zeros(5)
    UL = np.ascontiguousarray(UL, dtype=np.float64)
    UR = np.ascontiguousarray(UR, dtype=np.float64)
    r = lib.ns3d_debug_riemann(d, rs, GAMMA, UL.ctypes.data_as(_dp), UR.ctypes.data_as(_dp), F.ctypes.data_as(_dp))
    assert r == 0
    return F


def cons(rho, vel, p):
    vel = np.asarray(vel, dtype=np.float64)
    return np.array([rho, *(rho * vel), p / (GAMMA - 1) + 0.5 * rho * vel @ vel])


def physical_flux(U, d):
    rho, m, E = U[0], U[1:4], U[4]
    vel = m / rho
    p = (GAMMA - 1) * (E - 0.5 * rho * vel @ vel)
    un = vel[d]
    F = np.array([rho * un, *(rho * un * vel), (E + p) * un])
    F[1 + d] += p
    return F


def sw_split_reference(U, d, sign):
    """Steger & Warming (1981), 1-D split flux along the normal, with the
    tangential momentum and energy carried by the mass-flux weights."""
    rho, m, E = U[0], U[1:4], U[4]
    vel = m / rho
    p = (GAMMA - 1) * (E - 0.5 * rho * vel @ vel)
    c = np.sqrt(GAMMA * p / rho)
    un = vel[d]
    lam = np.array([un, un + c, un - c])
    lp = 0.5 * (lam + sign * np.abs(lam))
    n = np.zeros(3); n[d] = 1.0
    k = rho / (2 * GAMMA)
    vt2 = vel @ vel - un * un
    mass = 2 * (GAMMA - 1) * lp[0] + lp[1] + lp[2]
    mom = 2 * (GAMMA - 1) * lp[0] * vel + lp[1] * (vel + c * n) + lp[2] * (vel - c * n)
    W = (3 - GAMMA) * (lp[1] + lp[2]) * c * c / (2 * (GAMMA - 1))
    ene = (GAMMA - 1) * lp[0] * (un * un + vt2) + 0.5 * lp[1] * ((un + c) ** 2 + vt2) + \
        0.5 * lp[2] * ((un - c) ** 2 + vt2) + W
    return k * np.array([mass, *mom, ene])


def random_state(rng, mach=0.8):
    rho = rng.uniform(0.2, 2.0)
    p = rng.uniform(0.2, 3.0)
    c = np.sqrt(GAMMA * p / rho)
    return cons(rho, rng.uniform(-mach, mach, 3) * c, p)


@pytest.mark.parametrize("rs", range(7))
@pytest.mark.parametrize("d", range(3))
def test_consistency(lib, rs, d):
    rng = np.random.default_rng(10 * rs + d)
    for _ in range(50):
        U = random_state(rng, mach=2.0)
        F = flux(lib, d, rs, U, U)
        Fp = physical_flux(U, d)
        assert np.allclose(F, Fp, rtol=1e-12, atol=1e-12 * np.abs(Fp).max()), (rs, d, F, Fp)


@pytest.mark.parametrize("d", range(3))
def test_steger_warming_matches_published_split(lib, d):
    rng = np.random.default_rng(7 + d)
    for _ in range(200):
        UL, UR = random_state(rng, 1.5), random_state(rng, 1.5)
        ref = sw_split_reference(UL, d, +1) + sw_split_reference(UR, d, -1)
        F = flux(lib, d, 6, UL, UR)
        assert np.allclose(F, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max()), (F, ref)
        # the split parts of one state add up to its physical flux
        np.testing.assert_allclose(sw_split_reference(UL, d, +1) + sw_split_reference(UL, d, -1),
                                   physical_flux(UL, d), rtol=1e-12, atol=1e-12)


def test_steger_warming_upwinds_supersonic_flow(lib):
    rng = np.random.default_rng(3)
    for _ in range(50):
        rho, p = rng.uniform(0.5, 2), rng.uniform(0.5, 2)
        c = np.sqrt(GAMMA * p / rho)
        UL = cons(rho, [2.5 * c, 0.1, -0.2], p)
        UR = cons(rho * 1.3, [2.2 * c, 0.0, 0.3], p * 0.7)
        np.testing.assert_allclose(flux(lib, 0, 6, UL, UR), physical_flux(UL, 0), rtol=1e-12)
        np.testing.assert_allclose(flux(lib, 0, 6, UR * [1, -1, 1, 1, 1], UL * [1, -1, 1, 1, 1]),
                                   physical_flux(UL * [1, -1, 1, 1, 1], 0), rtol=1e-12)


def test_reference_solvers_match_oracle_known_answers(lib):
    """The six reference solvers evaluated by the library's host path agree with the
    oracle's restatement (pinned bit-for-bit to the reference) to rounding."""
    from oracle import oracle
    import os
    if not os.path.exists(oracle.PORT_LIB):
        oracle.build(ref=False)
    olib = C.CDLL(oracle.PORT_LIB)
    olib.orc_riemann.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double, _dp]
    rng = np.random.default_rng(11)
    for rs in range(6):
        for d in range(3):
            for _ in range(20):
                UL, UR = random_state(rng, 0.9), random_state(rng, 0.9)
                Fo = np.zeros(5)
                olib.orc_riemann(rs, UL.ctypes.data_as(_dp), UR.ctypes.data_as(_dp), d, GAMMA, Fo.ctypes.data_as(_dp))
                F = flux(lib, d, rs, UL, UR)
                assert np.allclose(F, Fo, rtol=1e-12, atol=1e-13 * np.abs(Fo).max()), (rs, d, F, Fo)
