"""Steger-Warming face flux on the GPU (this library's addition: the reference
declares the splitting but implements no formula, so there is no reference
output to match).  Checked as physics: Sod's shock tube with WENO5 against
the exact Riemann solution, beside Roe on the same grid, in both precisions."""
import math

import numpy as np
import pytest

from helpers import interior
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import shock_tube_state

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def exact_riemann(left, right, x, t, x0, g=GAMMA):
    """Exact solution of the 1-D Riemann problem (Newton iteration for p*,
    then sampling of the wave fan), density only."""
    (rl, ul, pl), (rr, ur, pr) = left, right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
            return (p - pk) * math.sqrt(A / (p + B)), math.sqrt(A / (B + p)) * (1 - (p - pk) / (2 * (B + p)))
        r = (p / pk) ** ((g - 1) / (2 * g))
        return 2 * ck / (g - 1) * (r - 1), 1 / (rk * ck) * (p / pk) ** (-(g + 1) / (2 * g))

    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(1e-8, p - dp)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = f(p, rl, pl, cl)
    fr, _ = f(p, rr, pr, cr)
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    rho = np.empty_like(x)
    for n, xi in enumerate(x):
        s = (xi - x0) / t
        if s <= us:  # left of the contact
            if p > pl:  # left shock
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * p / pl + (g - 1) / (2 * g))
                rho[n] = rl if s < sl else rl * (p / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pl + 1)
            else:
                csl = cl * (p / pl) ** ((g - 1) / (2 * g))
                if s < ul - cl:
                    rho[n] = rl
                elif s > us - csl:
                    rho[n] = rl * (p / pl) ** (1 / g)
                else:
                    rho[n] = rl * (2 / (g + 1) + (g - 1) / ((g + 1) * cl) * (ul - s)) ** (2 / (g - 1))
        else:
            if p > pr:  # right shock
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * p / pr + (g - 1) / (2 * g))
                rho[n] = rr if s > sr else rr * (p / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pr + 1)
            else:
                csr = cr * (p / pr) ** ((g - 1) / (2 * g))
                if s > ur + cr:
                    rho[n] = rr
                elif s < us + csr:
                    rho[n] = rr * (p / pr) ** (1 / g)
                else:
                    rho[n] = rr * (2 / (g + 1) - (g - 1) / ((g + 1) * cr) * (ur - s)) ** (2 / (g - 1))
    return rho


def run_tube(riemann, precision, nx=400, t_end=0.2, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    from ns3d_wcns_b200.solver import Solver
    P, G = make_params(n=(nx, 4, 4), L=(1.0, 1.0, 1.0), Ma=1.0, Re=math.inf, cfl=0.5, dt_fixed=-1.0,
                       interpolation=0, riemann=riemann, bcs=(3, 3, 0, 0, 0, 0), precision=precision)
    with Solver(P, G) as s:
        s.set_interior_primitives(*shock_tube_state(nx, 4, 4, left, right))
        t, steps = s.time_advance(t_end, 10 ** 5)
        assert abs(t - t_end) < 1e-12 and steps > 10
        W = interior(s.primitives())
    # the quasi-1-D solution is the same on every (j, k) line
    assert np.abs(W[:, :, :, :] - W[:, :1, :1, :]).max() < 1e-12
    return W[:, 0, 0, :]


@pytest.mark.parametrize("left,right", [((1.0, 0.0, 1.0), (0.125, 0.0, 0.1)),      # Sod
                                        ((0.445, 0.698, 3.528), (0.5, 0.0, 0.571))])  # Lax
def test_shock_tube_against_exact(gpu_lib, left, right):
    nx, t_end = 400, (0.2 if left[0] == 1.0 else 0.14)
    x = np.arange(nx) / nx
    ex = exact_riemann(left, right, x, t_end, x0=0.5 - 0.5 / nx)
    err = {}
    for rs in (6, 0):  # Steger-Warming, Roe
        W = run_tube(rs, 0, nx, t_end, left, right)
        err[rs] = float(np.mean(np.abs(W[0] - ex)))
    print("L1 density error: Steger-Warming %.3e, Roe %.3e" % (err[6], err[0]))
    assert err[6] < 1e-2 and err[6] < 2.0 * err[0], err
    # the mixed path follows the FP64 path with the same flux
    Wm = run_tube(6, 1, nx, t_end, left, right)
    W64 = run_tube(6, 0, nx, t_end, left, right)
    assert float(np.mean(np.abs(Wm[0] - W64[0]))) < 1e-4
