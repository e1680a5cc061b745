"""The reference's own C++ driver on the GPU path.

oracle/_ref/libns3d_dropin.so is the reference solver compiled from its
sources with range_kutta.cpp and timestep.cpp replaced by the drop-in
(ns3d_wcns_b200/compat/ns3d_gpu_compat.cpp: compute_rhs, runge_kutta_3 and
compute_timestep over the C ABI); oracle/_ref/libns3d_dropin_loop.so also
takes time_advance from the drop-in (maincycle.cpp left out: the state stays
on the GPU for the whole loop).  Running time_advance (maincycle.cpp:7-113)
through either must reproduce the CPU reference (oracle/_ref/libns3d_ref.so):
the conserved state, the temperature, the last stage's right-hand side that
runge_kutta_3 leaves in F.rhs_*, and the monitor values compute_diagnostics
and compute_total_energy leave in the Field3D.  The libraries are built where
the reference sources exist and travel as build products; the tests skip
where they are absent.
"""
import numpy as np
import pytest

from helpers import interior, rel_linf
from ns3d_wcns_b200.config import format_solver_in, make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state
from oracle import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.ref_available() and oracle.dropin_available()),
                                 reason="reference / drop-in libraries not built")]

CASES = ["iso_adaptive", "outflow_fixed", "iso_monitor_output"]


def _case(case):
    if case == "iso_adaptive":
        n = (16, 16, 16)
        P, G = make_params(n=n, Ma=0.3, Re=400.0, Pr=0.72, cfl=0.5, dt_fixed=-1.0, interpolation=3, riemann=2,
                           max_steps=6, TotalTime=0.02, output_Timefreq=1.0)
        st = isotropic_state(n, P.gamma, P.Ma, seed=4)
    elif case == "outflow_fixed":
        n = (14, 9, 8)
        P, G = make_params(n=n, L=(1.0, 0.7, 0.6), bcs=(3, 3, 1, 1, 0, 0), dt_fixed=2e-4, max_steps=4,
                           TotalTime=1.0, output_Timefreq=10.0, monitor_Stepfreq=2, monitor_res=True,
                           monitor_energy=True)
        st = random_state(n, seed=9, amp=0.2)
    else:
        # adaptive dt clipped to output times and to TotalTime, monitor every
        # 3 steps with residuals and energy, output writers called
        n = (16, 14, 12)
        P, G = make_params(n=n, L=(2 * np.pi, 1.75 * np.pi, 1.5 * np.pi), Ma=0.3, Re=400.0, Pr=0.72, cfl=0.5,
                           dt_fixed=-1.0, interpolation=3, riemann=2, max_steps=9, TotalTime=0.13,
                           output_Timefreq=0.05, monitor_Stepfreq=3, monitor_res=True, monitor_energy=True,
                           post_basicfield=True, isotropic_analyse=True)
        st = isotropic_state(n, P.gamma, P.Ma, seed=7)
    return P, G, st


def _run(lib_path, P, G, st):
    s = oracle.RefSolver(P, G, solver_in_text=format_solver_in(P, G), lib_path=lib_path)
    s.set_interior_prims(*st)
    s.time_advance()
    return s


def _compare(gpu, cpu, P):
    U, Ur = gpu.conserved(), cpu.conserved()
    assert max(rel_linf(a, b) for a, b in zip(U, Ur)) <= 1e-10
    assert rel_linf(gpu.get("T"), cpu.get("T")) <= 1e-10
    # runge_kutta_3 leaves its last stage's right-hand side in F.rhs_*
    R, Rr = interior(gpu.rhs()), interior(cpu.rhs())
    assert max(rel_linf(a, b) for a, b in zip(R, Rr)) <= 1e-10
    m, mr = gpu.monitor_values(), cpu.monitor_values()
    if P.monitor_energy:
        assert abs(m[0] - mr[0]) <= 1e-12 * abs(mr[0]), (m[0], mr[0])
    if P.monitor_res:
        assert np.all(np.abs(m[1:] - mr[1:]) <= 1e-9 * np.abs(mr[1:])), (m[1:], mr[1:])


@pytest.mark.parametrize("case", CASES)
def test_reference_time_advance_on_gpu(gpu_lib, case):
    """maincycle.cpp's own loop over the drop-in's runge_kutta_3 / compute_timestep."""
    P, G, st = _case(case)
    cpu = _run(oracle.REF_LIB, P, G, st)
    gpu = _run(oracle.DROPIN_LIB, P, G, st)
    _compare(gpu, cpu, P)


@pytest.mark.skipif(not oracle.os.path.exists(oracle.DROPIN_LOOP_LIB), reason="resident-loop drop-in not built")
@pytest.mark.parametrize("case", CASES)
def test_resident_time_advance_on_gpu(gpu_lib, case):
    """The drop-in's own time_advance: state resident on the GPU, residual
    norms and kinetic energy reduced on the device, the host Field3D refreshed
    before the output writers and at the end."""
    P, G, st = _case(case)
    cpu = _run(oracle.REF_LIB, P, G, st)
    gpu = _run(oracle.DROPIN_LOOP_LIB, P, G, st)
    _compare(gpu, cpu, P)
