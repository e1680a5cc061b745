"""Host checks of two rearrangements the fused RK stage relies on (no GPU).

1. The fused last stage keeps the largest wave speed s = |u| + a per block and
   divides once: for positive dx, min_i fl(dx / s_i) == fl(dx / max_i s_i) bit
   for bit, because correctly rounded division by a positive number is
   monotone.  numpy's float64 division is IEEE correctly rounded, like the
   device's.
2. The mixed path's increment form of runge_kutta_3 (range_kutta.cpp:53-91):
   U1 = U0 + D1, D1 = dt L0; U2 = U0 + D2, D2 = (D1 + dt L1) / 4;
   U3 = U0 + 2/3 (D2 + dt L2) -- the same combination as
   U2 = 3/4 U0 + 1/4 (U1 + dt L1), U3 = 1/3 U0 + 2/3 (U2 + dt L2), with the
   increments stored in FP32.  On a linear test system the two forms agree to
   FP32 rounding of the increments, far below the FP32 rounding of the state.
"""
import numpy as np


def test_cfl_min_of_quotients_equals_quotient_of_max():
    rng = np.random.default_rng(7)
    for trial in range(200):
        dx = float(rng.uniform(1e-3, 1.0))
        s = rng.uniform(0.1, 10.0, size=int(rng.integers(1, 4096)))
        if trial % 3 == 0:  # near-ties: speeds one ulp apart
            s[:2] = np.nextafter(s[0], np.inf), s[0]
        per_cell = np.min(dx / s)
        per_block = dx / np.max(s)
        assert per_cell == per_block


def test_cfl_nan_and_zero_speeds():
    # fmin / fmax skip NaN; a zero speed gives inf, capped at the reduction's 1e9
    s = np.array([np.nan, 2.0, 0.5])
    assert np.fmin.reduce(1.0 / s) == 1.0 / np.fmax.reduce(s)
    z = np.array([0.0, 0.0])
    with np.errstate(divide="ignore"):
        assert min(1e9, np.min(1.0 / z)) == min(1e9, 1.0 / np.max(z)) == 1e9


def _rhs(A, U):
    return A @ U


def test_rk3_increment_form_matches_standard_form():
    rng = np.random.default_rng(3)
    n = 64
    A = rng.standard_normal((n, n)) / np.sqrt(n) - 0.5 * np.eye(n)
    U0 = 1.0 + 0.1 * rng.standard_normal(n)
    dt = 0.01
    # standard SSP-RK3 in FP64
    U1 = U0 + dt * _rhs(A, U0)
    U2 = 0.75 * U0 + 0.25 * (U1 + dt * _rhs(A, U1))
    U3 = (1.0 / 3.0) * U0 + (2.0 / 3.0) * (U2 + dt * _rhs(A, U2))
    # increment form with FP32 increments
    D1 = np.float32(dt * _rhs(A, U0)).astype(np.float64)
    V1 = U0 + D1
    D2 = np.float32(0.25 * (D1 + dt * _rhs(A, V1))).astype(np.float64)
    V2 = U0 + D2
    V3 = U0 + (2.0 / 3.0) * (D2 + dt * _rhs(A, V2))
    # the increments are O(dt |L|): their FP32 rounding is ~1e-8 of them
    inc = np.max(np.abs(U3 - U0))
    assert np.max(np.abs(V3 - U3)) <= 1e-6 * inc
    # and far below the FP32 rounding of the state itself
    assert np.max(np.abs(V3 - U3)) < 0.1 * np.finfo(np.float32).eps * np.max(np.abs(U3))
