"""B200 (sm_100a) implementation of ns3d_wcns's RHS evaluation and RK3 time advance.

The product is libns3d_b200.so (C ABI in include/ns3d_b200.h, CUDA kernels in
csrc/); this package holds its build recipe and the Python host-side mirror of
the reference's interface (config.py: solver.in, solver.py: ns3d_func.h).
"""
from .config import (BCType, GridDesc, Interpolation, Precision, RiemannSolver, SolverParams,
                     format_solver_in, make_params, parse_solver_params, read_solver_params_from_file)

__all__ = ["BCType", "GridDesc", "Interpolation", "Precision", "RiemannSolver", "SolverParams",
           "format_solver_in", "make_params", "parse_solver_params", "read_solver_params_from_file"]
