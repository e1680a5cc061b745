"""Turbulence statistics of a state, on the host (or on a torch device).

Restatement of the reference's post-processing for decaying isotropic
turbulence, used to state the error of every reported statistic:

* ``energy_spectrum`` -- EnergySpectrum.cpp:63-135: FFT of u, v, w normalised
  by 1/N^3, E = (|u^|^2 + |v^|^2 + |w^|^2)/2 per mode, summed over shells
  k = lround(|k|) with signed wavenumbers k1 = i (i <= N/2) else i - N,
  Kmax = 2*NX.
* ``turbulence_stats`` -- ana_isotropic.cpp:230-305: mean mu(T) (Sutherland,
  field_structures.h:96-106), mean rho, nu = mean_mu / mean_rho, kinetic
  energy <|u|^2/2>, u_rms, and the dissipation eps = 2 nu sum_k k^2 E(k);
  plus ``total_energy`` = sum rho |u|^2 / 2 dV (postprocess.cpp:103-128).

These run off the hot path (the reference calls them at output times only).
Inputs are interior arrays in C order [k][j][i].
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np


def _torch():
    import torch
    return torch


def _t(x, device):
    """float64 torch tensor on `device` (zero-copy for a tensor already there)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64)
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=device)


def energy_spectrum(u, v, w, device: str = "cpu") -> np.ndarray:
    """Shell spectrum E(k), k = 0..2*NX (EnergySpectrum.cpp:63-135)."""
    torch = _torch()
    nz, ny, nx = u.shape
    N = nx * ny * nz
    er = None
    for f in (u, v, w):
        h = torch.fft.fftn(_t(f, device).contiguous()) / N
        e = (h.real * h.real + h.imag * h.imag)
        er = e if er is None else er + e
        del h
    er = er * 0.5

    def wav(n):
        i = torch.arange(n, device=device, dtype=torch.int64)
        return torch.where(i <= n // 2, i, i - n)

    k3, k2, k1 = wav(nz)[:, None, None], wav(ny)[None, :, None], wav(nx)[None, None, :]
    kk2 = (k1 * k1 + k2 * k2 + k3 * k3).to(torch.float64)
    # lround(sqrt(m)) for integer m: sqrt(m) is never a half integer, so floor(x + 0.5)
    shell = torch.floor(torch.sqrt(kk2) + 0.5).to(torch.int64)
    kmax = 2 * nx
    Ek = torch.zeros(kmax + 1, dtype=torch.float64, device=device)
    Ek.index_add_(0, shell.reshape(-1), er.reshape(-1))
    return Ek.cpu().numpy()


def sutherland_mu(T, mu0: float, S: float):
    """mu(T) = mu0 T^1.5 (1 + S)/(T + S) (field_structures.h:96-106)."""
    return mu0 * T ** 1.5 * (1.0 + S) / (T + S)


def turbulence_stats(rho, u, v, w, T, mu0: float, S: float, dV: float, device: str = "cpu") -> Dict:
    """Kinetic energy, u_rms, nu and the spectral dissipation of ana_isotropic.cpp:230-305.
    Inputs: numpy arrays or torch tensors (used in place when already on `device`)."""
    rho, u, v, w, T = (_t(x, device) for x in (rho, u, v, w, T))
    N = rho.numel()
    q = u * u + v * v + w * w
    mean_mu = float(sutherland_mu(T, mu0, S).sum()) / N
    mean_rho = float(rho.sum()) / N
    nu = mean_mu / mean_rho
    Ek = energy_spectrum(u, v, w, device)
    k = np.arange(Ek.size, dtype=np.float64)
    eps = float(np.sum(2.0 * nu * k * k * Ek))
    qs = float(q.sum())
    return {
        "total_energy": float(0.5 * (rho * q).sum()) * dV,    # postprocess.cpp:103-128
        "kinetic_energy": 0.5 * qs / N,                        # ana_isotropic.cpp:280
        "u_rms": math.sqrt(qs / (3.0 * N)),
        "mean_mu": mean_mu, "mean_rho": mean_rho, "nu": nu,
        "dissipation": eps, "spectrum": Ek,
    }


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2."""
    d = float(np.sqrt(np.sum((np.asarray(a, np.float64) - b) ** 2)))
    r = float(np.sqrt(np.sum(np.asarray(b, np.float64) ** 2)))
    return d / r if r > 0 else d
