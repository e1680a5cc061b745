"""Batched independent problems (ns3d_batch_* of the C ABI).

Many small ns3d_wcns runs of uneven size -- e.g. quasi-1D shock tubes on
Nx x 4 x 4 grids -- integrated to their own end times on one GPU, by the
wavefront schedule (every active problem one step per round of launches) or
one persistent cluster launch, whichever ``autotune`` measures faster; both
give the same bits for the compiled-in WENO5 + Roe scheme and agree to
rounding for the others.  Each problem follows time_advance's dt schedule with its
own CFL time step (maincycle.cpp:18-56).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _lib
from .config import GridDesc, SolverParams
from .solver import _params

_dp = C.POINTER(C.c_double)


class Batch:
    def __init__(self, P: SolverParams, grids: Sequence[GridDesc], t_end: Sequence[float], device: int = 0):
        self.lib = _lib.load()
        self.P = P
        self.grids = list(grids)
        n = len(self.grids)
        garr = (_lib.Grid * n)(*[_lib.Grid(g.global_nx, g.global_ny, g.global_nz, g.x0, g.y0, g.z0, g.Lx, g.Ly, g.Lz)
                                 for g in self.grids])
        te = np.ascontiguousarray(t_end, dtype=np.float64)
        h = C.c_void_p()
        r = self.lib.ns3d_batch_create(C.byref(_params(P, device, False)), n, garr, te.ctypes.data_as(_dp), C.byref(h))
        if r != 0:
            raise _lib.Ns3dError(r, self.lib.ns3d_status_string(r).decode())
        self.h = h

    def _check(self, r):
        if r != 0:
            raise _lib.Ns3dError(r, self.lib.ns3d_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ns3d_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_interior_primitives(self, i: int, rho, u, v, w, p) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, u, v, w, p)]
        t = (_dp * 5)(*[a.ctypes.data_as(_dp) for a in arrs])
        self._check(self.lib.ns3d_batch_set_interior_primitives(self.h, i, t))

    def run(self, max_steps: int = 10 ** 7) -> None:
        self._check(self.lib.ns3d_batch_run(self.h, int(max_steps)))

    def autotune(self, trial_steps: int = 20):
        """(cluster size, CTA width, resident CTAs per SM) of the fastest trial."""
        out = (C.c_int * 3)()
        self._check(self.lib.ns3d_batch_autotune(self.h, int(trial_steps), out))
        return out[0], out[1], out[2]

    def set_config(self, cluster: int, threads: int, ctas_per_sm: int = 1) -> None:
        self._check(self.lib.ns3d_batch_set_config(self.h, int(cluster), int(threads), int(ctas_per_sm)))

    def query(self, i: int):
        t, s, st = C.c_double(), C.c_int(), C.c_int()
        self._check(self.lib.ns3d_batch_query(self.h, i, C.byref(t), C.byref(s), C.byref(st)))
        return t.value, s.value, st.value

    def primitives(self, i: int) -> np.ndarray:
        g = self.grids[i]
        shp = (g.global_nz + 6, g.global_ny + 6, g.global_nx + 6)
        out = np.empty((5,) + shp)
        t = (_dp * 5)(*[out[q].ctypes.data_as(_dp) for q in range(5)])
        self._check(self.lib.ns3d_batch_download(self.h, i, t))
        return out


def shock_tube_problems(n: int = 512, seed: int = 0, sizes=(200, 400, 800, 1600), ny: int = 4, nz: int = 4):
    """Config-5 problem set: n quasi-1D shock tubes on [0,1] x [0,1]^2 with Nx
    drawn from ``sizes``; left/right (rho, u, p) drawn per problem from
    rho in [0.1,1], u in [-1,1], p in [0.1,3.5]; t_end in [0.14, 0.2]."""
    rng = np.random.default_rng(seed)
    nx = rng.choice(sizes, size=n)
    left = np.stack([rng.uniform(0.1, 1.0, n), rng.uniform(-1, 1, n), rng.uniform(0.1, 3.5, n)], axis=1)
    right = np.stack([rng.uniform(0.1, 1.0, n), rng.uniform(-1, 1, n), rng.uniform(0.1, 3.5, n)], axis=1)
    t_end = rng.uniform(0.14, 0.2, n)
    grids = [GridDesc(global_nx=int(x), global_ny=ny, global_nz=nz, Lx=1.0, Ly=1.0, Lz=1.0,
                      dx=1.0 / int(x), dy=1.0 / ny, dz=1.0 / nz) for x in nx]
    return grids, left, right, t_end
