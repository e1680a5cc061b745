"""ctypes front-end for the two CPU oracles (test infrastructure only).

* ``PortSolver`` -- the C restatement (oracle/ns3d_oracle.c, built into
  oracle/_build/libns3d_oracle.so).  Always available.
* ``RefSolver``  -- the unmodified reference sources compiled in place with
  single-rank stand-ins (oracle/_ref/libns3d_ref.so).  Available only where it
  has been built (it needs the reference sources at build time).

Both expose the same methods; arrays come back in Field3D layout
(idx3 = (k*sy + j)*sx + i, reshaped to [sz, sy, sx]).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "libns3d_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libns3d_ref.so")
DROPIN_LIB = os.path.join(HERE, "_ref", "libns3d_dropin.so")
DROPIN_LOOP_LIB = os.path.join(HERE, "_ref", "libns3d_dropin_loop.so")
# The reference sources (a checkout of ns3d_wcns): NS3D_REF_DIR, else a
# checkout named "reference" beside this repository.  Only the build of the
# test oracle reads them.
REF_SRC_DIR = os.path.abspath(os.environ.get("NS3D_REF_DIR") or
                              os.path.join(HERE, os.pardir, os.pardir, "reference"))

_dp = C.POINTER(C.c_double)


class OrcConfig(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("Ma", C.c_double), ("Re", C.c_double),
                ("cfl", C.c_double), ("dt_fixed", C.c_double), ("mdcd_diss", C.c_double),
                ("mdcd_disp", C.c_double), ("sutherland_s", C.c_double), ("Lx", C.c_double),
                ("Ly", C.c_double), ("Lz", C.c_double), ("nx", C.c_int), ("ny", C.c_int),
                ("nz", C.c_int), ("interpolation", C.c_int), ("riemann", C.c_int),
                ("char_recon", C.c_int), ("bc", C.c_int * 6)]


def build(ref: bool = True) -> None:
    """Compile the restatement, and the reference when its sources are present."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(REF_SRC_DIR):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_DIR={REF_SRC_DIR}"], check=True)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "ns3d_wcns_b200", "libns3d_b200.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin", f"REF_DIR={REF_SRC_DIR}"], check=True)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def dropin_available() -> bool:
    return os.path.exists(DROPIN_LIB)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class _Base:
    lib: C.CDLL

    def _shape(self):
        d = (C.c_int * 6)()
        self._dims(d)
        return list(d)

    def get(self, name: str) -> np.ndarray:
        nx, ny, nz = self.nx, self.ny, self.nz
        sx, sy, sz = nx + 6, ny + 6, nz + 6
        if name.startswith("flux_fx"):
            shape = (sz, sy, sx - 1)
        elif name.startswith("flux_fy"):
            shape = (sz, sy - 1, sx)
        elif name.startswith("flux_fz"):
            shape = (sz - 1, sy, sx)
        else:
            shape = (sz, sy, sx)
        out = np.empty(shape, dtype=np.float64)
        r = self._get(name.encode(), _ptr(out), C.c_long(out.size))
        if r < 0:
            raise KeyError(name)
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        r = self._set(name.encode(), _ptr(a), C.c_long(a.size))
        if r != 0:
            raise KeyError(f"{name}: {r}")

    def set_interior_prims(self, rho, u, v, w, p) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, w, p)]
        r = self._set_interior(*[_ptr(a) for a in arrs])
        if r != 0:
            raise RuntimeError("set_interior_prims failed")

    def conserved(self) -> np.ndarray:
        return np.stack([self.get(n) for n in ("rho", "rhou", "rhov", "rhow", "E")])

    def rhs(self) -> np.ndarray:
        return np.stack([self.get(n) for n in ("rhs_rho", "rhs_rhou", "rhs_rhov", "rhs_rhow", "rhs_E")])


class PortSolver(_Base):
    """The C restatement (oracle/ns3d_oracle.c)."""

    def __init__(self, P, G):
        if not os.path.exists(PORT_LIB):
            build(ref=False)
        lib = C.CDLL(PORT_LIB)
        lib.orc_init.argtypes = [C.POINTER(OrcConfig)]
        lib.orc_get.restype = C.c_long
        lib.orc_get.argtypes = [C.c_char_p, _dp, C.c_long]
        lib.orc_set.argtypes = [C.c_char_p, _dp, C.c_long]
        lib.orc_set_interior_prims.argtypes = [_dp] * 5
        lib.orc_rk3_step.argtypes = [C.c_double]
        lib.orc_timestep.restype = C.c_double
        lib.orc_total_energy.restype = C.c_double
        lib.orc_residuals.argtypes = [_dp]
        lib.orc_weno5.restype = C.c_double
        lib.orc_weno5.argtypes = [_dp]
        lib.orc_mdcd_linear.restype = C.c_double
        lib.orc_mdcd_linear.argtypes = [_dp, C.c_double, C.c_double]
        lib.orc_mdcd_hybrid.restype = C.c_double
        lib.orc_mdcd_hybrid.argtypes = [_dp, C.c_double, C.c_double]
        lib.orc_riemann.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double, _dp]
        self.lib = lib
        cfg = OrcConfig()
        cfg.gamma, cfg.Pr, cfg.Ma, cfg.Re = P.gamma, P.Pr, P.Ma, P.Re
        cfg.cfl, cfg.dt_fixed = P.cfl, P.dt_fixed
        cfg.mdcd_diss, cfg.mdcd_disp, cfg.sutherland_s = P.mdcd_diss, P.mdcd_disp, P.S_ref
        cfg.Lx, cfg.Ly, cfg.Lz = G.Lx, G.Ly, G.Lz
        cfg.nx, cfg.ny, cfg.nz = G.global_nx, G.global_ny, G.global_nz
        cfg.interpolation, cfg.riemann, cfg.char_recon = int(P.interpolation), int(P.riemann_solver), int(P.char_recon)
        for i, b in enumerate(P.bcs):
            cfg.bc[i] = int(b)
        r = lib.orc_init(C.byref(cfg))
        if r != 0:
            raise ValueError(f"oracle rejected the configuration ({r})")
        self.nx, self.ny, self.nz = G.global_nx, G.global_ny, G.global_nz
        self._get, self._set = lib.orc_get, lib.orc_set
        self._set_interior = lib.orc_set_interior_prims

    def compute_rhs(self): self.lib.orc_compute_rhs()
    def apply_boundary(self): self.lib.orc_apply_boundary()
    def rk3_step(self, dt: float): self.lib.orc_rk3_step(C.c_double(dt))
    def timestep(self) -> float: return self.lib.orc_timestep()
    def total_energy(self) -> float: return self.lib.orc_total_energy()

    def residuals(self) -> np.ndarray:
        out = np.zeros(5)
        self.lib.orc_residuals(_ptr(out))
        return out


class RefSolver(_Base):
    """The reference sources compiled in place (oracle/_ref/libns3d_ref.so)."""

    def __init__(self, P, G, solver_in_text: Optional[str] = None, lib_path: str = REF_LIB):
        from ns3d_wcns_b200.config import format_solver_in
        if not os.path.exists(lib_path):
            raise FileNotFoundError(lib_path)
        lib = C.CDLL(lib_path)
        lib.ref_init_file.argtypes = [C.c_char_p, C.c_double]
        lib.ref_get.argtypes = [C.c_char_p, _dp, C.c_long]
        lib.ref_set.argtypes = [C.c_char_p, _dp, C.c_long]
        lib.ref_set_interior_prims.argtypes = [_dp] * 5
        lib.ref_rk3_step.argtypes = [C.c_double]
        lib.ref_timestep.restype = C.c_double
        lib.ref_total_energy.restype = C.c_double
        lib.ref_params.argtypes = [_dp, C.POINTER(C.c_int)]
        lib.ref_residuals.argtypes = [_dp]
        lib.ref_monitor_values.argtypes = [_dp]
        self.lib = lib
        text = solver_in_text if solver_in_text is not None else format_solver_in(P, G)
        with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
            f.write(text)
            path = f.name
        try:
            r = lib.ref_init_file(path.encode(), C.c_double(P.S_ref))
        finally:
            os.unlink(path)
        if r != 0:
            raise RuntimeError("reference parser failed")
        self.nx, self.ny, self.nz = G.global_nx, G.global_ny, G.global_nz
        self._get, self._set = lib.ref_get, lib.ref_set
        self._set_interior = lib.ref_set_interior_prims

    def params(self):
        d = (C.c_double * 18)()
        i = (C.c_int * 16)()
        self.lib.ref_params(d, i)
        return list(d), list(i)

    def compute_rhs(self): self.lib.ref_compute_rhs()
    def apply_boundary(self): self.lib.ref_apply_boundary()
    def rk3_step(self, dt: float): self.lib.ref_rk3_step(C.c_double(dt))
    def timestep(self) -> float: return self.lib.ref_timestep()
    def total_energy(self) -> float: return self.lib.ref_total_energy()
    def time_advance(self): self.lib.ref_time_advance()

    def residuals(self) -> np.ndarray:
        out = np.zeros(5)
        self.lib.ref_residuals(_ptr(out))
        return out

    def initialize(self, kind: str) -> None:
        """initialize_riemann_2d / _sod_shock_tube / _uniform_field / _sine_x_field /
        init_isotropic_turbulence + ghost fill."""
        r = self.lib.ref_initialize({"riemann_2d": 0, "sod": 1, "uniform": 2, "sine_x": 3, "isotropic": 4}[kind])
        if r != 0:
            raise RuntimeError("ref_initialize failed")

    def monitor_values(self) -> np.ndarray:
        """F.global_Etot, F.global_res_rho ... F.global_res_E after time_advance."""
        out = np.zeros(6)
        self.lib.ref_monitor_values(_ptr(out))
        return out


def _kat_lib(path):
    lib = C.CDLL(path)
    pre = "ref_" if path == REF_LIB else "orc_"
    f_weno = getattr(lib, pre + "weno5")
    f_weno.restype = C.c_double
    f_weno.argtypes = [_dp]
    f_lin = getattr(lib, pre + "mdcd_linear")
    f_lin.restype = C.c_double
    f_lin.argtypes = [_dp, C.c_double, C.c_double]
    f_hyb = getattr(lib, pre + "mdcd_hybrid")
    f_hyb.restype = C.c_double
    f_hyb.argtypes = [_dp, C.c_double, C.c_double]
    f_rie = getattr(lib, pre + "riemann")
    f_rie.restype = None
    f_rie.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double, _dp]
    return f_weno, f_lin, f_hyb, f_rie


class Kernels:
    """Scalar interpolation / Riemann kernels of one oracle (port or reference)."""

    def __init__(self, which: str = "port"):
        if which == "port" and not os.path.exists(PORT_LIB):
            build(ref=False)
        self._w, self._l, self._h, self._r = _kat_lib(PORT_LIB if which == "port" else REF_LIB)

    def weno5(self, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        return self._w(_ptr(a))

    def mdcd_linear(self, f, disp, diss):
        a = np.ascontiguousarray(f, dtype=np.float64)
        return self._l(_ptr(a), disp, diss)

    def mdcd_hybrid(self, f, disp, diss):
        a = np.ascontiguousarray(f, dtype=np.float64)
        return self._h(_ptr(a), disp, diss)

    def riemann(self, solver, UL, UR, direction, gamma):
        a = np.ascontiguousarray(UL, dtype=np.float64)
        b = np.ascontiguousarray(UR, dtype=np.float64)
        out = np.zeros(5)
        self._r(int(solver), _ptr(a), _ptr(b), int(direction), float(gamma), _ptr(out))
        return out


def ref_isotropic(nx: int, ny: int, nz: int):
    """The reference's generate_full_turbulence (isotropic_ini.cpp:26-126) on an
    nx x ny x nz grid, from its generator's seed, as (u, v, w) arrays
    [nz, ny, nx] of the interior."""
    lib = C.CDLL(REF_LIB)
    lib.ref_isotropic_field.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
    out = [np.zeros(nx * ny * nz) for _ in range(3)]
    lib.ref_isotropic_field(nx, ny, nz, *[_ptr(a) for a in out])
    # reference order (i*ny + j)*nz + k -> [k][j][i]
    return tuple(np.ascontiguousarray(a.reshape(nx, ny, nz).transpose(2, 1, 0)) for a in out)
