"""The C restatement (oracle/) pinned to the reference.

* golden fixtures generated by the reference itself (tests/golden/, see
  make_golden.py): one RHS, a few RK3 steps, dt and kinetic energy for eight
  configurations covering every interpolation, Riemann solver, boundary type
  and characteristic interpolation -- the restatement must reproduce them
  bit for bit;
* scalar known answers of the interpolators and the six Riemann solvers;
* where the reference has been built here (oracle/_ref), extra live cases.
"""
import os

import numpy as np
import pytest

from helpers import golden_cases, interior, params_from_cfg
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = np.load(os.path.join(HERE, "golden", "ref_cases.npz"))
KATS = np.load(os.path.join(HERE, "golden", "kats.npz"))


@pytest.mark.parametrize("name,cfg", golden_cases(CASES), ids=[n for n, _ in golden_cases(CASES)])
def test_port_matches_reference_golden(name, cfg):
    P, G = params_from_cfg(cfg)
    s = oracle.PortSolver(P, G)
    s.set_interior_prims(*CASES[name + "_in"])
    s.compute_rhs()
    assert np.array_equal(interior(s.rhs()), CASES[name + "_rhs"], equal_nan=True)
    for _ in range(cfg["steps"]):
        s.rk3_step(cfg["dt"])
    assert np.array_equal(s.conserved(), CASES[name + "_U"], equal_nan=True)
    np.testing.assert_array_equal(s.timestep(), CASES[name + "_dt"])
    np.testing.assert_array_equal(s.total_energy(), CASES[name + "_ke"])


def test_port_scalar_kats():
    K = oracle.Kernels("port")
    st = KATS["kat_stencils"]
    assert np.array_equal([K.weno5(f) for f in st], KATS["kat_weno5"])
    assert np.array_equal([K.mdcd_linear(f, 0.0463783, 0.02) for f in st], KATS["kat_mdcd_linear"])
    assert np.array_equal([K.mdcd_hybrid(f, 0.0463783, 0.02) for f in st], KATS["kat_mdcd_hybrid"])
    F = KATS["kat_riemann"]
    for s in range(6):
        for d in range(3):
            got = np.array([K.riemann(s, UL, UR, d, 1.4) for UL, UR in KATS["kat_states"]])
            assert np.array_equal(got, F[s, d]), (s, d)


def test_kats_cover_both_mdcd_branches():
    # the hybrid detector must take both branches on the KAT stencils
    st = KATS["kat_stencils"]
    lin = KATS["kat_mdcd_linear"]
    hyb = KATS["kat_mdcd_hybrid"]
    assert np.sum(lin == hyb) > 0 and np.sum(lin != hyb) > 0
    assert len(st) == 64


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built in this container")
@pytest.mark.parametrize("interp,rs,ch,bcs", [
    (0, 2, 1, (0, 0, 3, 3, 1, 1)),
    (3, 0, 0, (4, 3, 2, 2, 0, 0)),
    (2, 5, 1, (3, 3, 3, 3, 3, 3)),
    (3, 4, 1, (0, 0, 0, 0, 0, 0)),
])
def test_port_matches_reference_live(interp, rs, ch, bcs):
    from ns3d_wcns_b200.config import make_params
    from ns3d_wcns_b200.initial import random_state
    n = (7, 6, 5)
    P, G = make_params(n=n, L=(1.0, 1.1, 0.7), interpolation=interp, riemann=rs, char_recon=ch, bcs=bcs)
    st = random_state(n, seed=interp * 10 + rs)
    a, b = oracle.PortSolver(P, G), oracle.RefSolver(P, G)
    a.set_interior_prims(*st)
    b.set_interior_prims(*st)
    for _ in range(2):
        a.rk3_step(2e-4)
        b.rk3_step(2e-4)
    assert np.array_equal(a.conserved(), b.conserved())
    assert np.array_equal(a.rhs(), b.rhs())
    # compute_diagnostics' residual norms of the last step
    assert np.array_equal(a.residuals(), b.residuals())
