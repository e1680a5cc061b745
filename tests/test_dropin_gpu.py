"""The reference's own C++ driver on the GPU path.

oracle/_ref/libns3d_dropin.so is the reference solver compiled from its
sources with range_kutta.cpp and timestep.cpp replaced by the drop-in
(ns3d_wcns_b200/compat/ns3d_gpu_compat.cpp: compute_rhs, runge_kutta_3 and
compute_timestep over the C ABI).  Running the reference's unmodified
time_advance (maincycle.cpp:7-113) through it must reproduce the CPU
reference (oracle/_ref/libns3d_ref.so) -- the integration a maintainer would
ship.  Both libraries are built where the reference sources exist and travel
as build products; the tests skip where they are absent.
"""
import numpy as np
import pytest

from helpers import rel_linf
from ns3d_wcns_b200.config import format_solver_in, make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state
from oracle import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.ref_available() and oracle.dropin_available()),
                                 reason="reference / drop-in libraries not built")]


@pytest.mark.parametrize("case", ["iso_adaptive", "outflow_fixed"])
def test_reference_time_advance_on_gpu(gpu_lib, case):
    if case == "iso_adaptive":
        n = (16, 16, 16)
        P, G = make_params(n=n, Ma=0.3, Re=400.0, Pr=0.72, cfl=0.5, dt_fixed=-1.0, interpolation=3, riemann=2,
                           max_steps=6, TotalTime=0.02, output_Timefreq=1.0)
        st = isotropic_state(n, P.gamma, P.Ma, seed=4)
    else:
        n = (14, 9, 8)
        P, G = make_params(n=n, L=(1.0, 0.7, 0.6), bcs=(3, 3, 1, 1, 0, 0), dt_fixed=2e-4, max_steps=4,
                           TotalTime=1.0, output_Timefreq=10.0)
        st = random_state(n, seed=9, amp=0.2)
    text = format_solver_in(P, G)
    cpu = oracle.RefSolver(P, G, solver_in_text=text)
    gpu = oracle.RefSolver(P, G, solver_in_text=text, lib_path=oracle.DROPIN_LIB)
    for s in (cpu, gpu):
        s.set_interior_prims(*st)
        s.time_advance()
    U, Ur = gpu.conserved(), cpu.conserved()
    assert max(rel_linf(a, b) for a, b in zip(U, Ur)) <= 1e-10
    T, Tr = gpu.get("T"), cpu.get("T")
    assert rel_linf(T, Tr) <= 1e-10
