"""Seeded synthetic initial conditions for the benchmark workloads.

Decaying isotropic turbulence on [0, 2*pi]^3 (periodic): a random solenoidal
velocity field with energy spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), scaled so
that u_rms = sqrt(<u^2+v^2+w^2>/3) equals the target (the u_rms definition of
ana_isotropic.cpp:280); rho = 1, T = 1, p = rho*Rgas*T = 1/(gamma Ma^2) as
isotropic_ini.cpp:184-186 sets them.  This generator is this build's own: the
reference's generator (isotropic_ini.cpp:25-127, k0=8, mt19937 seed 123) is
not used, and identical interior primitives are fed to the GPU path and the
oracle instead.

Arrays are returned in C order [k][j][i] (x fastest), the order of the
interior block of a Field3D array.
"""
from __future__ import annotations

import numpy as np


def isotropic_velocity(n, seed: int = 0, k0: float = 4.0, urms: float = 1.0):
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((3, nz, ny, nx))
    hat = np.fft.fftn(noise, axes=(1, 2, 3))
    kz = np.fft.fftfreq(nz, 1.0 / nz)[:, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kx = np.fft.fftfreq(nx, 1.0 / nx)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(k2)
    with np.errstate(divide="ignore", invalid="ignore"):
        Ek = kmag ** 4 * np.exp(-2.0 * (kmag / k0) ** 2)
        amp = np.where(k2 > 0, np.sqrt(Ek / (4.0 * np.pi * np.maximum(k2, 1e-30))), 0.0)
    hat *= amp[None]
    # solenoidal projection: u_hat -= k (k . u_hat) / |k|^2
    kdotu = kx * hat[0] + ky * hat[1] + kz * hat[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        f = np.where(k2 > 0, kdotu / np.maximum(k2, 1e-30), 0.0)
    hat[0] -= kx * f
    hat[1] -= ky * f
    hat[2] -= kz * f
    vel = np.real(np.fft.ifftn(hat, axes=(1, 2, 3)))
    vel -= vel.mean(axis=(1, 2, 3), keepdims=True)
    cur = np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2) / 3.0)
    vel *= urms / cur
    return vel[0].copy(), vel[1].copy(), vel[2].copy()


def isotropic_state(n, gamma: float, Ma: float, seed: int = 0, k0: float = 4.0, urms: float = 1.0):
    """Interior primitives (rho, u, v, w, p) for the isotropic workloads."""
    u, v, w = isotropic_velocity(n, seed, k0, urms)
    rho = np.ones_like(u)
    p = np.full_like(u, 1.0 / (gamma * Ma * Ma))
    return rho, u, v, w, p


def random_state(n, seed: int = 0, gamma: float = 1.4, Ma: float = 0.3, amp: float = 0.3):
    """Smooth-plus-noise random primitives for parity tests (all BCs, odd sizes)."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    p0 = 1.0 / (gamma * Ma * Ma)
    shp = (nz, ny, nx)
    rho = 1.0 + amp * 0.5 * rng.uniform(-1, 1, shp)
    u = amp * rng.uniform(-1, 1, shp) * 3.0
    v = amp * rng.uniform(-1, 1, shp) * 3.0
    w = amp * rng.uniform(-1, 1, shp) * 3.0
    p = p0 * (1.0 + amp * rng.uniform(-1, 1, shp))
    return rho, u, v, w, p


def shock_tube_state(nx: int, ny: int, nz: int, left, right, x_interface: float = 0.5, Lx: float = 1.0):
    """Quasi-1-D Riemann problem: (rho, u, p) left/right of x_interface, v = w = 0."""
    x = (np.arange(nx) + 0.0) * (Lx / nx)
    mask = (x < x_interface)[None, None, :]
    shp = (nz, ny, nx)
    rho = np.where(mask, left[0], right[0]) * np.ones(shp)
    u = np.where(mask, left[1], right[1]) * np.ones(shp)
    p = np.where(mask, left[2], right[2]) * np.ones(shp)
    z = np.zeros(shp)
    return rho, u, z.copy(), z.copy(), p
