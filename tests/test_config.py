"""solver.in contract: the host mirror parses like initialization.cpp:36-200."""
import math
import os
import tempfile

import pytest

from ns3d_wcns_b200.config import (BCType, Interpolation, Precision, RiemannSolver, ConfigError,
                                   format_solver_in, make_params, parse_solver_params,
                                   read_solver_params_from_file)
from oracle import oracle

TEXT = """
# comment line
Length_ref = 1.0
Re          = 500000
MA = 0.5
gamma       = 1.4
Pr          = 0.71
cfl         = 0.2
dt_fixed    = -0.0005
fvs_type       = LaxFriedrichs
interpolation  = mdcd_hybrid
vis_scheme     = C6th
char_recon     = TRUE
Riemann_Solver = HLLC_p
mdcd_disp = 0.0463783
mdcd_diss = 0.020
global_nx   = 64
global_ny   = 32
global_nz   = 6
bc_xmin = Outflow
bc_xmax = outflow
bc_ymin = wall
bc_ymax = Symmetry
bc_zmin = periodic
bc_zmax = Periodic
Lx = 2.0
Ly = 1.0
Lz = 0.5
max_steps = 10000
monitor_Stepfreq = 10
output_Timefreq = 0.1
TotalTime = 0.3
restart = Ture
restart_file = Field.h5
IsotropicAnalyse      = no
"""


def test_parse_known_answers():
    P, G, C = parse_solver_params(TEXT)
    assert P.Re == 500000 and P.Ma == 0.5 and P.cfl == 0.2 and P.dt_fixed == -0.0005
    assert P.interpolation == Interpolation.MDCD_HYBRID and P.char_recon is True
    assert P.riemann_solver == RiemannSolver.HLLC_p
    assert (G.global_nx, G.global_ny, G.global_nz) == (64, 32, 6)
    assert P.bcs == (BCType.Outflow, BCType.Outflow, BCType.Wall, BCType.Symmetry, BCType.Periodic,
                     BCType.Periodic)
    assert C.periods == (0, 0, 1)
    assert G.dx == 2.0 / 64 and G.dz == 0.5 / 6
    assert P.restart is True and P.restart_file == "Field.h5" and P.isotropic_analyse is False
    assert P.Rgas == 1.0 / (0.5 * 0.5 * 1.4) and P.mu == 1.0 / 500000
    assert P.Cv == 1.0 / (1.4 * (1.4 - 1.0) * 0.5 * 0.5) and P.Cp == P.Cv * 1.4
    assert P.ghost_layers == 3 and P.stencil == 6
    assert P.S_ref == 110.4 / 288.15


def test_unknown_bc_falls_back_to_periodic_and_zero_sets_one_ghost():
    P, G, C = parse_solver_params("bc_xmin = Nonsense\nbc_xmax = periodic\ninterpolation = zero\n")
    assert P.bc_xmin == BCType.Periodic and C.periods[0] == 1
    assert P.ghost_layers == 1 and P.stencil == 2


def test_build_keys():
    P, _, _ = parse_solver_params("sutherland_s = 0.5\nprecision = mixed\n")
    assert P.S_ref == 0.5 and P.precision == Precision.MIXED
    with pytest.raises(ConfigError):
        parse_solver_params("precision = fp16\n")


def test_roundtrip_and_file():
    P, G = make_params(n=(10, 12, 14), interpolation=2, riemann=5, char_recon=True, bcs=(3, 3, 1, 2, 0, 0))
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write(format_solver_in(P, G, extra=True))
    try:
        P2, G2, _ = read_solver_params_from_file(f.name)
    finally:
        os.unlink(f.name)
    assert P2.bcs == P.bcs and P2.interpolation == P.interpolation and G2.global_nz == 14
    with pytest.raises(FileNotFoundError):
        read_solver_params_from_file("/nonexistent/solver.in")


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built in this container")
def test_parser_matches_reference_parser():
    P, G, C = parse_solver_params(TEXT)
    r = oracle.RefSolver(P, G, solver_in_text=TEXT)
    d, i = r.params()
    mine_d = [P.gamma, P.Pr, P.Ma, P.Re, P.cfl, P.dt_fixed, P.mu, 110.4 / 288.15, P.Cv, P.Cp, P.Rgas,
              G.dx, G.dy, G.dz, P.mdcd_diss, P.mdcd_disp, P.TotalTime, P.output_Timefreq]
    # RefSolver overrides S_ref with P.S_ref (the reference value here)
    assert d == mine_d
    mine_i = [int(P.interpolation), int(P.riemann_solver), int(P.char_recon)] + list(P.bcs) + \
             [G.global_nx, G.global_ny, G.global_nz, P.max_steps, P.monitor_Stepfreq, int(P.fvs_type),
              int(P.vis_scheme)]
    assert i == mine_i
