"""solver.in configuration contract of ns3d_wcns, restated for the B200 build.

Mirrors ``read_solver_params_from_file`` (initialization.cpp:36-200) and the
``SolverParams`` / ``GridDesc`` structs (field_structures.h:33-186): same keys,
same case-insensitive matching, same defaults, same derived constants
(Cv, Cp, Rgas, mu, dx) and the same periodic-pair rule for ``periods``.

Additions of this build (opt-in keys the reference does not read):
  * ``sutherland_s`` -- Sutherland constant S/T_ref.  The reference hard-codes
    110.4/288.15 (field_structures.h:95); that stays the default.
  * ``precision = fp64 | mixed`` -- plain FP64 path (reference parity) or the
    mixed FP32/FP64 path.
"""
from __future__ import annotations

import dataclasses
import enum
import math
import os
from typing import Dict, Tuple


class Interpolation(enum.IntEnum):
    """Order as field_structures.h:131-136."""
    WENO5 = 0
    ZERO = 1
    MDCD_LINEAR = 2
    MDCD_HYBRID = 3


class RiemannSolver(enum.IntEnum):
    """Order as field_structures.h:137-144; StegerWarming is this build's
    addition (the reference declares the splitting, field_structures.h:113-119,
    but implements no formula)."""
    Roe = 0
    Rusanov = 1
    HLLC = 2
    HLL = 3
    HLLC_p = 4
    AUSM = 5
    StegerWarming = 6


class BCType(enum.IntEnum):
    """Order as field_structures.h:159."""
    Periodic = 0
    Wall = 1
    Symmetry = 2
    Outflow = 3
    Inflow = 4


class FVSType(enum.IntEnum):
    """Order as field_structures.h:113-118 (parsed, unused by the reference)."""
    StegerWarming = 0
    LaxFriedrichs = 1
    Rusanov = 2
    VanLeer = 3


class ViscousScheme(enum.IntEnum):
    """Order as field_structures.h:127-130 (parsed, unused by the reference)."""
    C6th = 0
    C4th = 1


class Precision(enum.IntEnum):
    FP64 = 0
    MIXED = 1


REFERENCE_S_REF = 110.4 / 288.15


@dataclasses.dataclass
class GridDesc:
    """field_structures.h:33-38."""
    global_nx: int = 16
    global_ny: int = 16
    global_nz: int = 16
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    Lx: float = 1.0
    Ly: float = 1.0
    Lz: float = 1.0
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0


@dataclasses.dataclass
class SolverParams:
    """field_structures.h:86-186 (defaults as the struct initialisers)."""
    gamma: float = 1.4
    Pr: float = 0.71
    Ma: float = 0.4
    Re: float = 500.0
    cfl: float = 0.1
    dt_fixed: float = -1.0
    mu: float = 1.0 / 500.0
    S_ref: float = REFERENCE_S_REF
    Cv: float = 1.0 / (1.4 * 0.4 * 0.4 * 0.4)
    Cp: float = 1.0 / (1.4 * 0.4 * 0.4 * 0.4) * 1.4
    Rgas: float = 1.0 / (0.4 * 0.4 * 1.4)
    fvs_type: FVSType = FVSType.StegerWarming
    interpolation: Interpolation = Interpolation.WENO5
    vis_scheme: ViscousScheme = ViscousScheme.C6th
    riemann_solver: RiemannSolver = RiemannSolver.Roe
    mdcd_diss: float = 0.01
    mdcd_disp: float = 0.0463783
    stencil: int = 6
    ghost_layers: int = 3
    char_recon: bool = False
    bc_xmin: BCType = BCType.Periodic
    bc_xmax: BCType = BCType.Periodic
    bc_ymin: BCType = BCType.Periodic
    bc_ymax: BCType = BCType.Periodic
    bc_zmin: BCType = BCType.Periodic
    bc_zmax: BCType = BCType.Periodic
    max_steps: int = 1
    monitor_Stepfreq: int = 1
    output_Timefreq: float = 1.0
    TotalTime: float = 1.0
    post_basicfield: bool = True
    isotropic_analyse: bool = True
    restart: bool = False
    restart_file: str = "field.h5"
    monitor_res: bool = True
    monitor_energy: bool = True
    # additions of this build
    precision: Precision = Precision.FP64

    @property
    def bcs(self) -> Tuple[int, int, int, int, int, int]:
        return (int(self.bc_xmin), int(self.bc_xmax), int(self.bc_ymin),
                int(self.bc_ymax), int(self.bc_zmin), int(self.bc_zmax))

    def get_mu(self, T: float) -> float:
        """Sutherland's law, field_structures.h:96-106."""
        return self.mu * T ** 1.5 * (1.0 + self.S_ref) / (T + self.S_ref)


@dataclasses.dataclass
class CartDecomp:
    """The part of field_structures.h:40-47 the parser writes (periods)."""
    periods: Tuple[int, int, int] = (0, 0, 0)


class ConfigError(ValueError):
    pass


def _parse_bool(v: str) -> bool:
    # initialization.cpp:30-34 (accepts the "ture" misspelling)
    return v.lower() in ("true", "ture", "yes", "1", "on")


def _stod(val: str) -> float:
    # std::stod parses the longest valid prefix; solver.in values are plain numbers
    try:
        return float(val.split()[0])
    except (ValueError, IndexError) as e:
        raise ConfigError(f"not a number: {val!r}") from e


def _stoi(val: str) -> int:
    try:
        return int(val.split()[0])
    except (ValueError, IndexError) as e:
        raise ConfigError(f"not an integer: {val!r}") from e


def _parse_bc(v: str) -> BCType:
    # initialization.cpp:134-140: unknown names fall back to Periodic
    return {"inflow": BCType.Inflow, "wall": BCType.Wall, "symmetry": BCType.Symmetry,
            "outflow": BCType.Outflow}.get(v, BCType.Periodic)


def parse_solver_params(text: str) -> Tuple[SolverParams, GridDesc, CartDecomp]:
    """Parse solver.in text exactly as initialization.cpp:36-200 does."""
    P = SolverParams()
    G = GridDesc()
    periods = [0, 0, 0]
    for raw in text.splitlines():
        line = raw.strip(" \t\r\n")
        if not line or line[0] == "#":
            continue
        eq = line.find("=")
        if eq < 0:
            continue
        key = line[:eq].strip(" \t\r\n")
        val = line[eq + 1:].strip(" \t\r\n")
        k, v = key.lower(), val.lower()
        if k == "gamma": P.gamma = _stod(val)
        elif k == "pr": P.Pr = _stod(val)
        elif k == "ma": P.Ma = _stod(val)
        elif k == "re": P.Re = _stod(val)
        elif k == "cfl": P.cfl = _stod(val)
        elif k == "dt_fixed": P.dt_fixed = _stod(val)
        elif k == "fvs_type":
            P.fvs_type = {"stegerwarming": FVSType.StegerWarming, "vanleer": FVSType.VanLeer,
                          "laxfriedrichs": FVSType.LaxFriedrichs}.get(v, P.fvs_type)
        elif k == "interpolation":
            P.interpolation = {"mdcd_hybrid": Interpolation.MDCD_HYBRID,
                               "mdcd_linear": Interpolation.MDCD_LINEAR,
                               "weno5": Interpolation.WENO5, "zero": Interpolation.ZERO}.get(v, P.interpolation)
        elif k == "vis_scheme":
            P.vis_scheme = {"c4": ViscousScheme.C4th, "c6": ViscousScheme.C6th}.get(v, P.vis_scheme)
        elif k == "char_recon": P.char_recon = v in ("yes", "true")
        elif k == "riemann_solver":
            P.riemann_solver = {"roe": RiemannSolver.Roe, "rusanov": RiemannSolver.Rusanov,
                                "hllc": RiemannSolver.HLLC, "hll": RiemannSolver.HLL,
                                "hllc_p": RiemannSolver.HLLC_p, "ausm": RiemannSolver.AUSM,
                                "steger_warming": RiemannSolver.StegerWarming,
                                "stegerwarming": RiemannSolver.StegerWarming}.get(v, P.riemann_solver)
        elif k == "mdcd_diss": P.mdcd_diss = _stod(val)
        elif k == "mdcd_disp": P.mdcd_disp = _stod(val)
        elif k == "global_nx": G.global_nx = _stoi(val)
        elif k == "global_ny": G.global_ny = _stoi(val)
        elif k == "global_nz": G.global_nz = _stoi(val)
        elif k == "x0": G.x0 = _stod(val)
        elif k == "y0": G.y0 = _stod(val)
        elif k == "z0": G.z0 = _stod(val)
        elif k == "lx": G.Lx = _stod(val)
        elif k == "ly": G.Ly = _stod(val)
        elif k == "lz": G.Lz = _stod(val)
        elif k == "max_steps": P.max_steps = _stoi(val)
        elif k == "monitor_stepfreq": P.monitor_Stepfreq = _stoi(val)
        elif k == "output_timefreq": P.output_Timefreq = _stod(val)
        elif k == "totaltime": P.TotalTime = _stod(val)
        elif k == "restart": P.restart = _parse_bool(val)
        elif k == "restart_file": P.restart_file = val
        # keys added by this build
        elif k == "sutherland_s": P.S_ref = _stod(val)
        elif k == "precision":
            if v not in ("fp64", "mixed"):
                raise ConfigError(f"precision must be fp64 or mixed, got {val!r}")
            P.precision = Precision.FP64 if v == "fp64" else Precision.MIXED
        # boundary keys form a separate if-chain in the reference (initialization.cpp:142-147)
        if k == "bc_xmin": P.bc_xmin = _parse_bc(v)
        elif k == "bc_xmax": P.bc_xmax = _parse_bc(v)
        elif k == "bc_ymin": P.bc_ymin = _parse_bc(v)
        elif k == "bc_ymax": P.bc_ymax = _parse_bc(v)
        elif k == "bc_zmin": P.bc_zmin = _parse_bc(v)
        elif k == "bc_zmax": P.bc_zmax = _parse_bc(v)
        elif k == "post_basicfield": P.post_basicfield = _parse_bool(val)
        elif k == "isotropicanalyse": P.isotropic_analyse = _parse_bool(val)
        elif k == "monitor_res": P.monitor_res = _parse_bool(val)
        elif k == "monitor_energy": P.monitor_energy = _parse_bool(val)
    # initialization.cpp:161-172
    if P.bc_xmin == BCType.Periodic and P.bc_xmax == BCType.Periodic: periods[0] = 1
    if P.bc_ymin == BCType.Periodic and P.bc_ymax == BCType.Periodic: periods[1] = 1
    if P.bc_zmin == BCType.Periodic and P.bc_zmax == BCType.Periodic: periods[2] = 1
    G.dx = G.Lx / G.global_nx
    G.dy = G.Ly / G.global_ny
    G.dz = G.Lz / G.global_nz
    # initialization.cpp:175-192
    if P.interpolation == Interpolation.ZERO:
        P.ghost_layers, P.stencil = 1, 2
    else:
        P.ghost_layers, P.stencil = 3, 6
    # initialization.cpp:194-197
    P.Cv = 1.0 / (P.gamma * (P.gamma - 1.0) * P.Ma * P.Ma)
    P.Cp = P.Cv * P.gamma
    P.Rgas = 1.0 / (P.Ma * P.Ma * P.gamma)
    P.mu = 1.0 / P.Re
    return P, G, CartDecomp(tuple(periods))


def read_solver_params_from_file(fname: str) -> Tuple[SolverParams, GridDesc, CartDecomp]:
    """initialization.cpp:36-47: raises FileNotFoundError where the reference returns false."""
    with open(fname, "r") as f:
        return parse_solver_params(f.read())


_ENUM_NAMES = {
    Interpolation.WENO5: "WENO5", Interpolation.ZERO: "ZERO",
    Interpolation.MDCD_LINEAR: "MDCD_LINEAR", Interpolation.MDCD_HYBRID: "MDCD_HYBRID",
}


def format_solver_in(P: SolverParams, G: GridDesc, extra: bool = False) -> str:
    """Write a solver.in that both the reference parser and this one read back
    to the same parameters.  ``extra`` adds this build's own keys."""
    fmt = lambda x: repr(float(x))
    lines = [
        f"gamma = {fmt(P.gamma)}", f"Pr = {fmt(P.Pr)}", f"Ma = {fmt(P.Ma)}", f"Re = {fmt(P.Re)}",
        f"cfl = {fmt(P.cfl)}", f"dt_fixed = {fmt(P.dt_fixed)}",
        f"interpolation = {_ENUM_NAMES[Interpolation(P.interpolation)]}",
        f"char_recon = {'True' if P.char_recon else 'False'}",
        f"Riemann_Solver = {RiemannSolver(P.riemann_solver).name}",
        f"mdcd_disp = {fmt(P.mdcd_disp)}", f"mdcd_diss = {fmt(P.mdcd_diss)}",
        f"global_nx = {G.global_nx}", f"global_ny = {G.global_ny}", f"global_nz = {G.global_nz}",
        f"x0 = {fmt(G.x0)}", f"y0 = {fmt(G.y0)}", f"z0 = {fmt(G.z0)}",
        f"Lx = {fmt(G.Lx)}", f"Ly = {fmt(G.Ly)}", f"Lz = {fmt(G.Lz)}",
        f"max_steps = {P.max_steps}", f"monitor_Stepfreq = {P.monitor_Stepfreq}",
        f"output_Timefreq = {fmt(P.output_Timefreq)}", f"TotalTime = {fmt(P.TotalTime)}",
        f"restart = False",
    ]
    names = ["bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax", "bc_zmin", "bc_zmax"]
    for n, b in zip(names, P.bcs):
        lines.append(f"{n} = {BCType(b).name}")
    tf = lambda b: "True" if b else "False"
    lines += [f"Post_BasicField = {tf(P.post_basicfield)}", f"IsotropicAnalyse = {tf(P.isotropic_analyse)}",
              f"monitor_Res = {tf(P.monitor_res)}", f"monitor_Energy = {tf(P.monitor_energy)}"]
    if extra:
        lines.append(f"sutherland_s = {fmt(P.S_ref)}")
        lines.append(f"precision = {'fp64' if P.precision == Precision.FP64 else 'mixed'}")
    return "\n".join(lines) + "\n"


def make_params(n=(32, 32, 32), L=(2 * math.pi,) * 3, gamma=1.4, Pr=0.72, Ma=0.3, Re=100.0,
                cfl=0.5, dt_fixed=1e-3, interpolation=Interpolation.WENO5,
                riemann=RiemannSolver.Roe, char_recon=False, bcs=(BCType.Periodic,) * 6,
                S_ref=110.4 / 273.15, mdcd_disp=0.0463783, mdcd_diss=0.01,
                precision=Precision.FP64, **kw) -> Tuple[SolverParams, GridDesc]:
    """Convenience constructor returning (P, G) with derived constants filled as
    the parser would (round-trips through format_solver_in)."""
    P = SolverParams()
    G = GridDesc(global_nx=n[0], global_ny=n[1], global_nz=n[2], Lx=L[0], Ly=L[1], Lz=L[2])
    P.gamma, P.Pr, P.Ma, P.Re, P.cfl, P.dt_fixed = gamma, Pr, Ma, Re, cfl, dt_fixed
    P.interpolation, P.riemann_solver, P.char_recon = Interpolation(interpolation), RiemannSolver(riemann), bool(char_recon)
    P.mdcd_disp, P.mdcd_diss = mdcd_disp, mdcd_diss
    (P.bc_xmin, P.bc_xmax, P.bc_ymin, P.bc_ymax, P.bc_zmin, P.bc_zmax) = [BCType(b) for b in bcs]
    # output and monitoring off unless asked for
    P.post_basicfield = P.isotropic_analyse = P.monitor_res = P.monitor_energy = False
    for k, v in kw.items():
        setattr(P, k, v)
    P2, G2, _ = parse_solver_params(format_solver_in(P, G))
    P2.S_ref = S_ref
    P2.precision = Precision(precision)
    return P2, G2
