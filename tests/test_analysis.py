"""Host statistics (spectrum, dissipation) against closed-form answers."""
import math

import numpy as np

from ns3d_wcns_b200 import analysis


def _grid(n):
    x = 2 * math.pi * np.arange(n) / n
    return np.meshgrid(x, x, x, indexing="ij")  # [k][j][i] -> z, y, x


def test_spectrum_single_mode():
    n = 16
    z, y, x = _grid(n)
    u = np.sin(3 * x)
    zero = np.zeros_like(u)
    Ek = analysis.energy_spectrum(u, zero, zero)
    assert Ek.size == 2 * n + 1
    # <u^2>/2 = 1/4, all of it in shell 3
    assert abs(Ek[3] - 0.25) < 1e-14 and abs(Ek.sum() - 0.25) < 1e-14


def test_spectrum_parseval_and_shells():
    n = 12
    rng = np.random.default_rng(1)
    u, v, w = rng.standard_normal((3, n, n, n))
    Ek = analysis.energy_spectrum(u, v, w)
    assert abs(Ek.sum() - 0.5 * np.mean(u * u + v * v + w * w)) < 1e-12
    # shell of mode (i,j,k) = (5,3,2): sqrt(38) = 6.16 -> 6; (4,4,4): sqrt(48) = 6.93 -> 7
    z, y, x = _grid(n)
    f = np.cos(5 * x + 3 * y + 2 * z)
    Ek = analysis.energy_spectrum(f, 0 * f, 0 * f)
    assert abs(Ek[6] - 0.25) < 1e-13
    f = np.cos(4 * x + 4 * y + 4 * z)
    Ek = analysis.energy_spectrum(f, 0 * f, 0 * f)
    assert abs(Ek[7] - 0.25) < 1e-13


def test_dissipation_single_mode():
    n = 16
    z, y, x = _grid(n)
    u = np.sin(2 * y)
    zero = np.zeros_like(u)
    rho = np.ones_like(u)
    T = np.full_like(u, 1.3)
    mu0, S = 1.0 / 400.0, 110.4 / 273.15
    st = analysis.turbulence_stats(rho, u, zero, zero, T, mu0, S, dV=(2 * math.pi / n) ** 3)
    nu = mu0 * 1.3 ** 1.5 * (1 + S) / (1.3 + S)
    assert abs(st["nu"] / nu - 1) < 1e-14
    # eps = 2 nu k^2 E(k), E(2) = 1/4
    assert abs(st["dissipation"] / (2 * nu * 4 * 0.25) - 1) < 1e-12
    assert abs(st["total_energy"] / (0.25 * (2 * math.pi) ** 3) - 1) < 1e-12
    assert abs(st["u_rms"] - math.sqrt(0.5 / 3)) < 1e-14
