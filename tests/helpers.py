"""Shared helpers of the parity tests."""
from __future__ import annotations

import json

import numpy as np

from ns3d_wcns_b200.config import make_params


def rel_linf(a, b) -> float:
    """max|a-b| / max|b| (relative L-infinity)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def rel_linf_per_var(a, b):
    return [rel_linf(x, y) for x, y in zip(a, b)]


def interior(x):
    return x[..., 3:-3, 3:-3, 3:-3]


def golden_cases(npz):
    names = sorted({k[:-4] for k in npz.files if k.endswith("_cfg")})
    out = []
    for n in names:
        cfg = json.loads(bytes(npz[n + "_cfg"]).decode())
        out.append((n, cfg))
    return out


def params_from_cfg(cfg):
    P, G = make_params(n=tuple(cfg["n"]), L=tuple(cfg["L"]), interpolation=cfg["interpolation"],
                       riemann=cfg["riemann"], char_recon=cfg["char_recon"], bcs=tuple(cfg["bcs"]),
                       Ma=cfg["Ma"], Re=cfg["Re"], Pr=cfg["Pr"])
    P.S_ref = cfg["S_ref"]
    return P, G
