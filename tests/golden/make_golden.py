"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run in a container that has the reference sources (it builds oracle/_ref from
them): ``python tests/golden/make_golden.py``.  The fixtures pin the C
restatement (oracle/ns3d_oracle.c) bit-for-bit and travel with the repository
to machines without the reference sources.

Contents of ref_cases.npz, per case <c>:
  <c>_cfg        json of the solver.in parameters
  <c>_in         interior primitives (5, nz, ny, nx)
  <c>_rhs        one compute_rhs after apply_boundary + p2c, interior (5, nz, ny, nx)
  <c>_U          conserved state after the case's RK3 steps, full Field3D arrays
  <c>_dt, <c>_ke compute_timestep / compute_total_energy of that state
kats.npz: scalar known answers of weno5 / mdcd_linear / mdcd_hybrid and the
six Riemann solvers on seeded stencils and states.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ns3d_wcns_b200.config import make_params  # noqa: E402
from ns3d_wcns_b200.initial import isotropic_state, random_state  # noqa: E402
from oracle import oracle  # noqa: E402

P, O, W, S, I = 0, 3, 1, 2, 4  # boundary types
CASES = [
    # name, n, interp, riemann, char, bcs, steps, dt, init
    ("weno_roe_per", (6, 5, 4), 0, 0, 0, (P,) * 6, 2, 1e-3, "random"),
    ("hyb_hllc_per", (6, 5, 4), 3, 2, 0, (P,) * 6, 2, 1e-3, "random"),
    ("lin_hll_char", (6, 5, 4), 2, 3, 1, (P,) * 6, 2, 1e-3, "random"),
    ("weno_rus_out", (7, 5, 4), 0, 1, 0, (O,) * 6, 2, 5e-4, "random"),
    ("weno_hllcp_wall", (5, 6, 4), 0, 4, 0, (W, W, S, S, O, O), 2, 5e-4, "random"),
    ("hyb_ausm_inflow", (6, 4, 5), 3, 5, 0, (I, O, P, P, W, S), 2, 5e-4, "random"),
    ("weno_roe_halfper", (6, 5, 4), 0, 0, 1, (P, O, W, P, S, I), 1, 5e-4, "random"),
    ("iso8_weno_roe", (8, 8, 8), 0, 0, 0, (P,) * 6, 3, 1e-3, "isotropic"),
]


def run_case(name, n, interp, rs, ch, bcs, steps, dt, init, out):
    L = (2 * np.pi,) * 3 if init == "isotropic" else (1.0, 0.8, 0.9)
    Pm, G = make_params(n=n, L=L, interpolation=interp, riemann=rs, char_recon=ch, bcs=bcs,
                        Ma=0.3, Re=100.0, Pr=0.72)
    st = isotropic_state(n, Pm.gamma, Pm.Ma, seed=3) if init == "isotropic" else random_state(n, seed=7)
    ref = oracle.RefSolver(Pm, G)
    ref.set_interior_prims(*st)
    ref.compute_rhs()
    rhs = ref.rhs()[:, 3:-3, 3:-3, 3:-3]
    for _ in range(steps):
        ref.rk3_step(dt)
    cfg = dict(n=n, L=L, interpolation=interp, riemann=rs, char_recon=ch, bcs=bcs, steps=steps, dt=dt,
               Ma=0.3, Re=100.0, Pr=0.72, S_ref=Pm.S_ref)
    out[name + "_cfg"] = np.frombuffer(json.dumps(cfg).encode(), dtype=np.uint8)
    out[name + "_in"] = np.stack(st)
    out[name + "_rhs"] = rhs
    out[name + "_U"] = ref.conserved()
    out[name + "_dt"] = np.array(ref.timestep())
    out[name + "_ke"] = np.array(ref.total_energy())


def kats(out):
    rng = np.random.default_rng(11)
    K = oracle.Kernels("ref")
    st = []
    for t in range(64):
        kind = t % 4
        if kind == 0:
            f = 1.0 + 0.1 * rng.standard_normal(6)
        elif kind == 1:
            f = np.where(np.arange(6) < rng.integers(1, 6), 1.0, 0.125) + 1e-3 * rng.standard_normal(6)
        elif kind == 2:
            f = np.full(6, rng.uniform(0.5, 20))
        else:
            f = 20.0 + rng.standard_normal(6)
        st.append(f)
    st = np.array(st)
    out["kat_stencils"] = st
    out["kat_weno5"] = np.array([K.weno5(f) for f in st])
    out["kat_mdcd_linear"] = np.array([K.mdcd_linear(f, 0.0463783, 0.02) for f in st])
    out["kat_mdcd_hybrid"] = np.array([K.mdcd_hybrid(f, 0.0463783, 0.02) for f in st])
    states = []
    for t in range(48):
        rl, rr = rng.uniform(0.1, 1.5, 2)
        vl, vr = rng.uniform(-1.5, 1.5, (2, 3)) * (3.0 if t % 3 == 0 else 1.0)
        pl, pr = rng.uniform(0.1, 3.5, 2)
        g = 1.4
        UL = np.r_[rl, rl * vl, pl / (g - 1) + 0.5 * rl * vl @ vl]
        UR = np.r_[rr, rr * vr, pr / (g - 1) + 0.5 * rr * vr @ vr]
        states.append(np.stack([UL, UR]))
    states = np.array(states)
    out["kat_states"] = states
    F = np.zeros((6, 3, len(states), 5))
    for s in range(6):
        for d in range(3):
            for t, (UL, UR) in enumerate(states):
                F[s, d, t] = K.riemann(s, UL, UR, d, 1.4)
    out["kat_riemann"] = F


def main():
    oracle.build(ref=True)
    out = {}
    for c in CASES:
        run_case(*c, out=out)
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **out)
    k = {}
    kats(k)
    np.savez_compressed(os.path.join(HERE, "kats.npz"), **k)
    print("wrote", sorted(out)[:3], "...", os.path.getsize(os.path.join(HERE, "ref_cases.npz")), "bytes")


if __name__ == "__main__":
    main()
