"""Host-side mirror of the reference's hot-path interface over the C ABI.

``Solver`` owns one device handle (libns3d_b200.so) for one grid.  The
module-level functions carry the reference's names and argument meaning
(ns3d_func.h): they take a host ``Field3D`` (numpy arrays in the reference's
SoA ghost-cell layout), run the step on the GPU and write the results back
into the host arrays, as a C++ host calling the C ABI would.

There is no CPU fallback: without the built library or a CUDA device every
call raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib
from .config import GridDesc, Precision, SolverParams

_dp = C.POINTER(C.c_double)

CONSERVED = ("rho", "rhou", "rhov", "rhow", "E")
PRIMITIVE = ("rho", "u", "v", "w", "p")
RHS = ("rhs_rho", "rhs_rhou", "rhs_rhov", "rhs_rhow", "rhs_E")


def _params(P: SolverParams, device: int, check_state: bool, keep_rhs: bool = False) -> _lib.Params:
    lib = _lib.load()
    p = _lib.Params()
    lib.ns3d_params_default(C.byref(p))
    p.gamma, p.Pr, p.Ma, p.Re = P.gamma, P.Pr, P.Ma, P.Re
    p.cfl, p.dt_fixed = P.cfl, P.dt_fixed
    p.mdcd_diss, p.mdcd_disp, p.sutherland_s = P.mdcd_diss, P.mdcd_disp, P.S_ref
    p.interpolation, p.riemann_solver, p.char_recon = int(P.interpolation), int(P.riemann_solver), int(P.char_recon)
    for i, b in enumerate(P.bcs):
        p.bc[i] = int(b)
    p.precision = int(P.precision)
    p.device = device
    p.check_state = int(check_state)
    p.keep_rhs = int(keep_rhs)
    return p


class Solver:
    """One GPU-resident ns3d_wcns state (whole domain on one device)."""

    def __init__(self, P: SolverParams, G: GridDesc, device: int = 0, check_state: bool = False,
                 keep_rhs: bool = False):
        self.lib = _lib.load()
        self.P, self.G = P, G
        self.device = device
        grid = _lib.Grid(G.global_nx, G.global_ny, G.global_nz, G.x0, G.y0, G.z0, G.Lx, G.Ly, G.Lz)
        h = C.c_void_p()
        r = self.lib.ns3d_create(C.byref(_params(P, device, check_state, keep_rhs)), C.byref(grid), C.byref(h))
        if r != 0:
            raise _lib.Ns3dError(r, self.lib.ns3d_last_error(None).decode() or
                                 self.lib.ns3d_status_string(r).decode())
        self.h = h
        d = (C.c_int * 3)()
        self.lib.ns3d_field_dims(h, d)
        self.sx, self.sy, self.sz = d[0], d[1], d[2]
        self.shape = (self.sz, self.sy, self.sx)

    # -- plumbing
    def _check(self, r: int) -> None:
        if r != 0:
            raise _lib.Ns3dError(r, self.lib.ns3d_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ns3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _ptrs(arrs: Sequence[np.ndarray]):
        t = (_dp * len(arrs))()
        for i, a in enumerate(arrs):
            t[i] = a.ctypes.data_as(_dp)
        return t

    # -- state transfer
    def upload_primitives(self, fields: Sequence[np.ndarray]) -> None:
        """Full Field3D arrays (rho,u,v,w,p), ghosts as given."""
        arrs = [np.ascontiguousarray(f, dtype=np.float64).reshape(-1) for f in fields]
        for a in arrs:
            if a.size != self.sx * self.sy * self.sz:
                raise ValueError("expected Field3D-sized arrays")
        self._check(self.lib.ns3d_upload_primitives(self.h, self._ptrs(arrs)))

    def set_interior_primitives(self, rho, u, v, w, p) -> None:
        """Interior (nz,ny,nx) primitives, then the device ghost fill."""
        n = self.G.global_nx * self.G.global_ny * self.G.global_nz
        arrs = [np.ascontiguousarray(f, dtype=np.float64).reshape(-1) for f in (rho, u, v, w, p)]
        for a in arrs:
            if a.size != n:
                raise ValueError("expected interior-sized arrays")
        self._check(self.lib.ns3d_set_interior_primitives(self.h, self._ptrs(arrs)))

    INIT_KINDS = {"riemann_2d": 0, "sod": 1, "uniform": 2, "sine_x": 3, "isotropic": 4}

    def initialize(self, kind: str) -> None:
        """One of the reference's built-in initialisers on the device, then the
        ghost fill (main.cpp:85-99): riemann_2d, sod, uniform, sine_x or
        isotropic (init_isotropic_turbulence, isotropic_ini.cpp:131-193)."""
        self._check(self.lib.ns3d_initialize(self.h, self.INIT_KINDS[kind]))

    def download(self, what: int) -> np.ndarray:
        nq = 1 if what == _lib.NS3D_TEMPERATURE else 5
        out = np.empty((nq,) + self.shape, dtype=np.float64)
        self._check(self.lib.ns3d_download(self.h, what, self._ptrs([out[q] for q in range(nq)])))
        return out[0] if nq == 1 else out

    def primitives(self) -> np.ndarray: return self.download(_lib.NS3D_PRIMITIVE)
    def conserved(self) -> np.ndarray: return self.download(_lib.NS3D_CONSERVED)
    def rhs(self) -> np.ndarray: return self.download(_lib.NS3D_RHS)
    def temperature(self) -> np.ndarray: return self.download(_lib.NS3D_TEMPERATURE)

    # -- the hot path
    def apply_boundary(self) -> None: self._check(self.lib.ns3d_apply_boundary(self.h))
    def compute_rhs(self) -> None: self._check(self.lib.ns3d_compute_rhs(self.h))
    def rk3_step(self, dt: float) -> None: self._check(self.lib.ns3d_rk3_step(self.h, C.c_double(dt)))

    def rk3_steps(self, nsteps: int, dt: float) -> None:
        self._check(self.lib.ns3d_rk3_steps(self.h, int(nsteps), C.c_double(dt)))

    def residuals(self) -> np.ndarray:
        """compute_diagnostics' residual norms of the last step (F.global_res_rho ... F.global_res_E)."""
        out = (C.c_double * 5)()
        self._check(self.lib.ns3d_residuals(self.h, out))
        return np.array(list(out))

    def compute_timestep(self) -> float:
        x = C.c_double()
        self._check(self.lib.ns3d_compute_timestep(self.h, C.byref(x)))
        return x.value

    def total_energy(self) -> float:
        x = C.c_double()
        self._check(self.lib.ns3d_total_energy(self.h, C.byref(x)))
        return x.value

    def diagnostics(self) -> Dict[str, float]:
        x = (C.c_double * 6)()
        self._check(self.lib.ns3d_diagnostics(self.h, x))
        return {"kinetic_energy": x[0], "grad_u_sq": x[1], "mean_mu": x[2], "mean_rho": x[3],
                "dissipation": x[4], "u_rms": x[5]}

    def time_advance(self, t_end: float, max_steps: int, time: float = 0.0):
        t = C.c_double(time)
        n = C.c_int(0)
        r = self.lib.ns3d_time_advance(self.h, C.c_double(t_end), int(max_steps), C.byref(t), C.byref(n))
        self._check(r)
        return t.value, n.value

    def synchronize(self) -> None: self._check(self.lib.ns3d_synchronize(self.h))

    def launches(self) -> int:
        x = C.c_long()
        self.lib.ns3d_last_launch_count(self.h, C.byref(x))
        return x.value

    # -- adjoint
    def vjp_rhs(self, rbar: np.ndarray) -> np.ndarray:
        """(dR/dU)^T rbar at the current state; rbar (5, sz, sy, sx)."""
        rb = [np.ascontiguousarray(rbar[q], dtype=np.float64) for q in range(5)]
        out = np.zeros((5,) + self.shape)
        self._check(self.lib.ns3d_vjp_rhs(self.h, self._ptrs(rb), self._ptrs([out[q] for q in range(5)])))
        return out

    def vjp_rk3_step(self, dt: float, ubar_next: np.ndarray) -> np.ndarray:
        ub = [np.ascontiguousarray(ubar_next[q], dtype=np.float64) for q in range(5)]
        out = np.zeros((5,) + self.shape)
        self._check(self.lib.ns3d_vjp_rk3_step(self.h, C.c_double(dt), self._ptrs(ub),
                                               self._ptrs([out[q] for q in range(5)])))
        return out

    def adjoint_kinetic_energy(self, nsteps: int, dt: float, checkpoint_every: int = 20):
        """(J, grad (3, nz, ny, nx), stats dict) -- see ns3d_adjoint_kinetic_energy."""
        n = (self.G.global_nz, self.G.global_ny, self.G.global_nx)
        grad = np.zeros((3,) + n)
        J = C.c_double()
        st = (C.c_double * 4)()
        self._check(self.lib.ns3d_adjoint_kinetic_energy(self.h, int(nsteps), C.c_double(dt), int(checkpoint_every),
                                                         C.byref(J), self._ptrs([grad[q] for q in range(3)]), st))
        return J.value, grad, {"forward_ms": st[0], "adjoint_ms": st[1], "adjoint_bytes": st[2],
                               "recomputed_steps": st[3]}

    def profile(self, enable: bool = True) -> None:
        self._check(self.lib.ns3d_profile(self.h, int(enable)))

    def profile_report(self) -> Dict[str, Dict[str, float]]:
        buf = C.create_string_buffer(1 << 14)
        self._check(self.lib.ns3d_profile_report(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms = line.split()
            out[name] = {"launches": int(n), "ms": float(ms)}
        return out

    def device_fields(self, what: int):
        ptrs = (C.c_void_p * 5)()
        lay = (C.c_long * 6)()
        self._check(self.lib.ns3d_device_fields(self.h, what, ptrs, lay))
        return [ptrs[i] for i in range(5)], list(lay)

    def device_view(self, what: int):
        """Zero-copy torch views (5, sz, sy, sx) of a device-resident group
        (ghost-inclusive Field3D extents; the padding is skipped by strides)."""
        import torch
        ptrs, (sx, sy, sz, px, off, esz) = self.device_fields(what)
        typestr = "<f8" if esz == 8 else "<f4"

        class _Iface:
            def __init__(self, ptr):
                self.__cuda_array_interface__ = {
                    "shape": (sz, sy, sx), "typestr": typestr, "data": (ptr + off * esz, False),
                    "strides": (sy * px * esz, px * esz, esz), "version": 2}

        return [torch.as_tensor(_Iface(p), device=f"cuda:{self.device}") for p in ptrs]

    def turbulence_stats(self) -> Dict:
        """Turbulence statistics of the current state computed on the GPU from
        the resident fields (analysis.turbulence_stats: kinetic energy, u_rms,
        nu, spectrum E(k) and dissipation 2 nu sum k^2 E(k), as the
        reference's EnergySpectrum.cpp / ana_isotropic.cpp), FP64."""
        from . import analysis
        self.synchronize()
        if int(self.P.precision) == int(Precision.MIXED):
            rho, m1, m2, m3, E = (x[3:-3, 3:-3, 3:-3].double() for x in self.device_view(_lib.NS3D_CONSERVED))
            u, v, w = m1 / rho, m2 / rho, m3 / rho
            p = (self.P.gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v + w * w))
        else:
            rho, u, v, w, p = (x[3:-3, 3:-3, 3:-3] for x in self.device_view(_lib.NS3D_PRIMITIVE))
        Rgas = 1.0 / (self.P.gamma * self.P.Ma * self.P.Ma)
        T = p / (rho * Rgas)
        dV = (self.G.Lx / self.G.global_nx) * (self.G.Ly / self.G.global_ny) * (self.G.Lz / self.G.global_nz)
        mu0 = 0.0 if self.P.Re == float("inf") else 1.0 / self.P.Re
        return analysis.turbulence_stats(rho, u, v, w, T, mu0, self.P.S_ref, dV, device=f"cuda:{self.device}")

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        self._check(self.lib.ns3d_set_stream(self.h, C.c_void_p(stream_ptr or 0)))


# ---------------------------------------------------------------------------
# Reference-named entry points over a host Field3D (ns3d_func.h)
# ---------------------------------------------------------------------------

class Field3D:
    """Host arrays in the reference layout (field_structures.h:196-373): each
    of shape (sz, sy, sx), idx3 = (k*sy + j)*sx + i."""

    def __init__(self, G: GridDesc, ng: int = 3):
        self.nx, self.ny, self.nz = G.global_nx, G.global_ny, G.global_nz
        self.sx, self.sy, self.sz = self.nx + 2 * ng, self.ny + 2 * ng, self.nz + 2 * ng
        shp = (self.sz, self.sy, self.sx)
        for n in CONSERVED + ("u", "v", "w", "p", "T") + RHS + ("rho0", "rhou0", "rhov0", "rhow0", "E0"):
            setattr(self, n, np.zeros(shp))
        self.rho[...] = 1.0  # Field3D::allocate
        self._solver: Optional[Solver] = None

    def attach(self, solver: Solver) -> "Field3D":
        self._solver = solver
        return self

    def _push(self) -> Solver:
        s = self._solver
        if s is None:
            raise RuntimeError("Field3D is not attached to a Solver")
        s.upload_primitives([self.rho, self.u, self.v, self.w, self.p])
        return s

    def _pull(self, s: Solver, rhs: bool = False) -> None:
        W = s.primitives()
        U = s.conserved()
        self.rho[...] = W[0]; self.u[...] = W[1]; self.v[...] = W[2]; self.w[...] = W[3]; self.p[...] = W[4]
        self.rhou[...] = U[1]; self.rhov[...] = U[2]; self.rhow[...] = U[3]; self.E[...] = U[4]
        self.T[...] = s.temperature()
        if rhs:
            R = s.rhs()
            for n, a in zip(RHS, R):
                getattr(self, n)[...] = a


def apply_boundary(F: Field3D, G=None, C_=None, P=None) -> None:
    """apply_boundary (boundary.cpp:14-54) followed by the state round trip."""
    s = F._push(); s.apply_boundary(); F._pull(s)


def compute_rhs(F: Field3D, C_=None, G=None, P=None, out_reqs=None) -> None:
    """compute_rhs (range_kutta.cpp:11-43): fills F.rhs_*."""
    s = F._push(); s.compute_rhs(); F._pull(s, rhs=True)


def runge_kutta_3(F: Field3D, C_=None, G=None, P=None, out_reqs=None, dt: float = 0.0) -> None:
    """recordConservedTo0 + runge_kutta_3 (range_kutta.cpp:46-92)."""
    s = F._push()
    for a, b in zip(("rho0", "rhou0", "rhov0", "rhow0", "E0"), CONSERVED):
        getattr(F, a)[...] = getattr(F, b)
    s.rk3_step(dt)
    F._pull(s, rhs=True)


def compute_timestep(F: Field3D, G=None, P=None) -> float:
    """compute_timestep (timestep.cpp:5-23)."""
    return F._push().compute_timestep()


def compute_total_energy(F: Field3D, G=None, C_=None, P=None) -> float:
    """compute_total_energy (postprocess.cpp:103-128); returns global_Etot."""
    return F._push().total_energy()
