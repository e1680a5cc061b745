#!/usr/bin/env python
"""Benchmark of the ns3d_wcns RK3 step on B200: cell-updates/s.

Workload (the GPU drop-in configuration): decaying isotropic turbulence on a
periodic 256^3 grid over [0, 2pi]^3, seeded solenoidal field with
E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, u_rms = 1, rho = 1, T = 1, Ma = 0.3,
Re = 400, Pr = 0.72, S/T_ref = 110.4/273.15, MDCD_HYBRID interpolation + HLLC
flux, 6th-order viscous terms, SSP-RK3 with the adaptive CFL = 0.5 time step
of compute_timestep.  One step = compute_timestep + one full RK3 step (three
RHS evaluations), exactly the work time_advance does per step.  Synthetic
inputs: seeded by rank; the reference publishes no dataset.

  value       device-timed whole-job cell-updates/s (state resident in HBM,
              plain FP64 path: the reference's arithmetic), K steps of
              ns3d_time_advance (the dt schedule on the device, steps in
              CUDA graphs)
  e2e         the same through the C ABI with host Field3D buffers, as the
              drop-in's time_advance runs it: the primitive state uploaded
              from pinned host memory at the start, then per step
              ns3d_compute_timestep (dt read back) + ns3d_rk3_step, every 10th
              step the monitor (ns3d_residuals + ns3d_total_energy read back),
              and the state downloaded to the host at the end -- all inside
              the timed region; e2e_full_state: every step uploads the state
              and downloads it again (a host that keeps its Field3D current
              after every step)
  mixed       the mixed FP32/FP64 path on the same workload
  grid_512    both paths at 512^3 (the mixed-precision config's larger grid)
  roofline    the dominant kernel's achieved algorithmic GB/s over its
              CUDA-event launch time vs the measured HBM copy bandwidth
  cpu_baseline the reference solver compiled from its sources (oracle/_ref),
              one host core, bounded 64^3 sample of the same scheme

N > 1 GPUs (torchrun): the 256^3 domain decomposed into N z-slabs, one per
GPU (strong scaling), halos exchanged by NCCL point-to-point operations after
every RK stage; max-over-ranks device time.
``--impl reference`` times the reference's CPU implementation on the host
cores (one single-rank process per core on 32^3 samples).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "isotropic turbulence 256^3 periodic, MDCD_HYBRID + HLLC, Ma 0.3, Re 400, CFL 0.5 adaptive"
METRIC = "cell-updates/s at 256^3 (RK3 step incl. CFL dt), plain FP64 GPU path; mixed FP32/FP64 reported alongside"


def bench_params(n: int, precision: int = 0):
    from ns3d_wcns_b200.config import make_params
    import math
    return make_params(n=(n, n, n), L=(2 * math.pi,) * 3, Ma=0.3, Re=400.0, Pr=0.72, cfl=0.5, dt_fixed=-1.0,
                       interpolation=3, riemann=2, S_ref=110.4 / 273.15, precision=precision)


# --------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (clock, power, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    PERIOD_MS = 50

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []  # (host arrival time, csv line)
        self.t_begin = self.t_end = None

    def start(self):
        """Start sampling and wait for the first sample, so that the timed
        region that follows is covered from its start."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", str(self.PERIOD_MS), "-i", str(self.device)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.monotonic()
        while not self.lines and self.proc.poll() is None and time.monotonic() - t0 < 10:
            time.sleep(0.01)

    def begin(self):
        self.t_begin = time.monotonic()

    def end(self):
        self.t_end = time.monotonic()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples that arrived inside the timed region (plus one period for the read latency)
        lo = self.t_begin if self.t_begin is not None else -math.inf
        hi = self.t_end + self.PERIOD_MS * 1e-3 if self.t_end is not None else math.inf
        for t, ln in self.lines:
            if not lo <= t <= hi:
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); smax.append(float(f[2])); power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "power_w_max": max(power), "samples": len(sm)}


# --------------------------------------------------------------- CPU baseline

def _cpu_worker(args):
    """One single-rank reference (or port) process: steps of the bench scheme."""
    n, steps, warmup, seed = args
    sys.path.insert(0, ROOT)
    from ns3d_wcns_b200.initial import isotropic_state
    from oracle import oracle
    P, G = bench_params(n)
    if oracle.ref_available():
        s, kind = oracle.RefSolver(P, G), "reference"
    else:
        s, kind = oracle.PortSolver(P, G), "port"
    s.set_interior_prims(*isotropic_state((n, n, n), P.gamma, P.Ma, seed=seed))
    for _ in range(warmup):
        s.rk3_step(s.timestep())
    t0 = time.perf_counter()
    for _ in range(steps):
        s.rk3_step(s.timestep())
    return time.perf_counter() - t0, kind


def cpu_baseline(n=64, steps=4):
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1) as pool:
        dt, kind = pool.map(_cpu_worker, [(n, steps, 0, 0)])[0]
    return {"value": n ** 3 * steps / dt, "unit": "cell-updates/s", "cores": 1, "kind": kind,
            "sample": f"{n}^3 periodic, same scheme (MDCD_HYBRID+HLLC, adaptive CFL), {steps} RK3 steps, "
                      f"{dt:.1f} s on one host core"}


def run_reference(args, rank):
    """--impl reference: the reference's CPU path on all host cores (rank 0 only)."""
    if rank != 0:
        return
    import multiprocessing as mp
    from oracle import oracle
    oracle.build(ref=os.path.isdir(oracle.REF_SRC_DIR))
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    n = 32
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(n, args.steps, args.warmup, r) for r in range(cores)])
    wall = time.perf_counter() - t0
    times = [r[0] for r in res]
    kind = res[0][1]
    value = cores * n ** 3 * args.steps / max(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * max(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{n}^3 per process", "processes": cores,
                   "mpi": "reference MPI build unavailable on this box (no mpicxx, MPI runtime, FFTW or HDF5 in "
                          "the image): single-rank reference processes, one per host core"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                         "sample": f"{cores} single-rank processes x {n}^3 periodic, {args.steps} timed steps each "
                                   f"(reference has no threads; replicas bound its MPI scaling), wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- adjoint

def adjoint_report(device: int, n: int = 64, nsteps: int = 200, dt: float = 2e-3, ce: int = 20, ndir: int = 16,
                   interp: int = 0, riemann: int = 0, fd: bool = True):
    """Config 4: 64^3 isotropic, Re 200, dt 2e-3, 200 RK3 steps, checkpoint every 20;
    gradient of the final kinetic energy w.r.t. the initial velocity, checked
    against central finite differences (h = 1e-6) on ndir seeded directions.
    interp / riemann: WENO5 + Roe (0, 0), MDCD_LINEAR + HLLC (2, 2), or the
    benchmark scheme MDCD_HYBRID + HLLC (3, 2) with fd=False: its detector is
    a switch, and over 200 steps at 64^3 perturbations of 1e-6 flip enough
    faces that central differences are not derivatives (measured: the h and
    2h differences disagree by 450 %), so only its cost is reported; its VJPs
    are checked against finite differences over one RHS and one step
    (tests/test_adjoint_gpu.py)."""
    import numpy as np
    import math
    from ns3d_wcns_b200.config import make_params
    from ns3d_wcns_b200.initial import isotropic_state
    from ns3d_wcns_b200.solver import Solver
    P, G = make_params(n=(n, n, n), L=(2 * math.pi,) * 3, Ma=0.3, Re=200.0, Pr=0.72, dt_fixed=dt,
                       interpolation=interp, riemann=riemann, S_ref=110.4 / 273.15)
    st = isotropic_state((n, n, n), P.gamma, P.Ma, seed=4)
    rng = np.random.default_rng(16)
    with Solver(P, G, device=device) as s:
        s.set_interior_primitives(*st)
        s.rk3_steps(3, dt)  # warm-up
        s.set_interior_primitives(*st)
        J, grad, stats = s.adjoint_kinetic_energy(nsteps, dt, ce)
        s.set_interior_primitives(*st)
        J2, grad2, stats2 = s.adjoint_kinetic_energy(nsteps, dt, ce)  # warm timing
        # the plain forward pass of the same steps (no checkpoint copies), device-timed
        # on the handle's stream
        import torch
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.set_interior_primitives(*st)
        s.rk3_steps(2, dt)
        s.set_interior_primitives(*st)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.rk3_steps(nsteps, dt)
        e1.record(stream)
        torch.cuda.synchronize()
        plain_forward_ms = e0.elapsed_time(e1)
        errs, errs4, noise, errsn = [], [], [], []
        gnorm = float(np.sqrt(np.sum(grad2 * grad2)))
        h = 1e-6

        def J_at(eps, d):
            rho, u, v, w, p = st
            s.set_interior_primitives(rho, u + eps * d[0], v + eps * d[1], w + eps * d[2], p)
            s.rk3_steps(nsteps, dt)
            return s.total_energy()

        for _ in range(ndir if fd else 0):
            d = rng.standard_normal((3, n, n, n))
            d /= np.sqrt(np.mean(d * d))
            Jp1, Jm1, Jp2, Jm2 = J_at(h, d), J_at(-h, d), J_at(2 * h, d), J_at(-2 * h, d)
            fd = (Jp1 - Jm1) / (2 * h)              # central difference, h = 1e-6
            fd2 = (Jp2 - Jm2) / (4 * h)             # the same with 2h
            fd4 = (4 * fd - fd2) / 3                # fourth-order combination
            ad = float(np.sum(grad2 * d))
            errs.append(abs(fd - ad) / abs(fd))
            errs4.append(abs(fd4 - ad) / abs(fd4))
            errsn.append(abs(fd - ad) / (gnorm * float(np.sqrt(np.sum(d * d)))))
            noise.append(abs(fd - fd2) / abs(fd))   # size of the FD's own error
    scheme = {(0, 0): "WENO5+Roe", (3, 2): "MDCD_HYBRID+HLLC", (2, 2): "MDCD_LINEAR+HLLC"}.get((interp, riemann))
    if not fd:
        return {"config": f"{n}^3 isotropic {scheme}, Re 200, dt {dt}, {nsteps} steps, checkpoint every {ce}",
                "J": J2, "forward_ms": stats2["forward_ms"], "adjoint_ms": stats2["adjoint_ms"],
                "plain_forward_ms": plain_forward_ms,
                "adjoint_over_plain_forward": stats2["adjoint_ms"] / plain_forward_ms,
                "fd": "not a derivative over this horizon (detector switches); VJPs checked over one RHS / step"}
    return {"config": f"{n}^3 isotropic {scheme}, Re 200, dt {dt}, {nsteps} steps, checkpoint every {ce}",
            "J": J2, "forward_ms": stats2["forward_ms"], "adjoint_ms": stats2["adjoint_ms"],
            "adjoint_over_forward": stats2["adjoint_ms"] / stats2["forward_ms"],
            "plain_forward_ms": plain_forward_ms,
            "adjoint_over_plain_forward": stats2["adjoint_ms"] / plain_forward_ms,
            "peak_adjoint_bytes": stats2["adjoint_bytes"], "fd_directions": ndir, "fd_h": 1e-6,
            "fd_max_rel_err": max(errs), "fd_median_rel_err": float(np.median(errs)),
            "fd4_max_rel_err": max(errs4), "fd4_median_rel_err": float(np.median(errs4)),
            "fd_h_vs_2h_max_rel": max(noise),
            "fd_max_err_over_grad_norm": max(errsn),  # |fd - ad| / (|grad| |d|)
            "recomputed_steps": stats2["recomputed_steps"],
            "forward_pass_includes": "checkpoint copies and the last segment's stage-state copies; "
                                     "plain_forward_ms: ns3d_rk3_steps of the same steps without them"}


# --------------------------------------------------------------- batched

def _ref_tube(args):
    """CPU run of one shock tube (spawned process): the reference compiled from
    its sources (oracle/_ref) or the C restatement pinned bit for bit to it.
    Returns the final primitives, the wall seconds and the steps."""
    nx, left, right, t_end, which = args
    sys.path.insert(0, ROOT)
    import math
    from ns3d_wcns_b200.config import make_params
    from ns3d_wcns_b200.initial import shock_tube_state
    from oracle import oracle
    P, G = make_params(n=(nx, 4, 4), L=(1.0, 1.0, 1.0), Ma=1.0, Re=math.inf, cfl=0.5, dt_fixed=-1.0,
                       interpolation=0, riemann=0, bcs=(3, 3, 0, 0, 0, 0))
    use_ref = which == "reference" and oracle.ref_available()
    s = oracle.RefSolver(P, G) if use_ref else oracle.PortSolver(P, G)
    s.set_interior_prims(*shock_tube_state(nx, 4, 4, left, right))
    t, steps = 0.0, 0
    t0 = time.perf_counter()
    while abs(t_end - t) > 1e-12:
        dt = s.timestep()
        if t + dt > t_end:
            dt = t_end - t
        if dt <= 1e-12:
            break
        t += dt
        s.rk3_step(dt)
        steps += 1
        if t >= t_end:
            break
    wall = time.perf_counter() - t0
    import numpy as np
    return np.stack([s.get(k) for k in ("rho", "u", "v", "w", "p")]), wall, steps, \
        ("reference" if use_ref else "port")


def batched_report(device: int, n: int = 512, check=((200, 8, "reference"), (400, 2, "port"))):
    """Config 5: n quasi-1D shock tubes Nx x 4 x 4, Nx in {200,400,800,1600}, seeded left/right
    states, t_end in [0.14, 0.2], inviscid WENO5+Roe, CFL 0.5, x Outflow, y/z Periodic; one
    persistent launch (autotuned, CUDA graph).  Per-instance relative L1 error against CPU runs
    of the first `count` problems of each checked Nx (the reference, or the C restatement pinned
    bit for bit to it), and a CPU problems/s baseline: the reference's measured per-core rate on
    the Nx = 200 sample, applied to the whole batch's cell-updates on all host cores."""
    import math
    import multiprocessing as mp
    import numpy as np
    from ns3d_wcns_b200.batch import Batch, shock_tube_problems
    from ns3d_wcns_b200.config import make_params
    from ns3d_wcns_b200.initial import shock_tube_state
    P, _ = make_params(n=(8, 4, 4), Ma=1.0, Re=math.inf, cfl=0.5, dt_fixed=-1.0, interpolation=0, riemann=0,
                       bcs=(3, 3, 0, 0, 0, 0))
    grids, left, right, t_end = shock_tube_problems(n, seed=5)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    with Batch(P, grids, t_end, device=device) as b:
        for i, g in enumerate(grids):
            b.set_interior_primitives(i, *shock_tube_state(g.global_nx, 4, 4, left[i], right[i]))
        cfg = b.autotune(trial_steps=30)
        for i, g in enumerate(grids):  # fresh start after tuning
            b.set_interior_primitives(i, *shock_tube_state(g.global_nx, 4, 4, left[i], right[i]))
        t0 = time.perf_counter()
        b.run()
        wall = time.perf_counter() - t0
        steps = [b.query(i)[1] for i in range(n)]
        cell_updates = sum(g.global_nx * 16 * s for g, s in zip(grids, steps))
        jobs, idx = [], []
        for nx, count, which in check:
            sel = [i for i, g in enumerate(grids) if g.global_nx == nx][:count]
            idx += sel
            jobs += [(nx, tuple(left[i]), tuple(right[i]), float(t_end[i]), which) for i in sel]
        # longest tubes first, one job at a time, so that the pool's wall time
        # is close to the longest single run
        order = sorted(range(len(jobs)), key=lambda j: -jobs[j][0])
        with mp.get_context("spawn").Pool(min(len(jobs), cores)) as pool:
            done = pool.map(_ref_tube, [jobs[j] for j in order], chunksize=1)
        refs = [None] * len(jobs)
        for j, r in zip(order, done):
            refs[j] = r
        per_nx, rate = {}, []
        for i, (Wr, sec, st, kind) in zip(idx, refs):
            Wg = b.primitives(i)
            sl = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))
            l1 = float(np.abs(Wg[sl] - Wr[sl]).sum() / np.abs(Wr[sl]).sum())
            nx = grids[i].global_nx
            e = per_nx.setdefault(f"Nx{nx}_{kind}", {"count": 0, "l1": []})
            e["count"] += 1
            e["l1"].append(l1)
            if kind == "reference" and nx == 200:
                rate.append(nx * 16 * st / sec)
        for e in per_nx.values():
            e["max_l1"], e["median_l1"] = max(e["l1"]), float(np.median(e["l1"]))
            del e["l1"]
    cpu = None
    if rate:
        per_core = float(np.median(rate))
        cpu_wall = cell_updates / (per_core * cores)
        cpu = {"problems_per_s": n / cpu_wall, "unit": "problems/s", "cores": cores, "kind": "reference",
               "sample": f"{len(rate)} Nx=200 tubes run concurrently, one per core: median {per_core:.3g} "
                         f"cell-updates/s per core, applied to the batch's {cell_updates:.3g} cell-updates "
                         f"(the GPU run's step counts) on {cores} cores"}
    return {"config": f"{n} shock tubes Nx x 4 x 4, Nx in {{200,400,800,1600}}, WENO5+Roe, CFL 0.5, t_end 0.14-0.2",
            "problems_per_s": n / wall, "wall_s": wall, "cell_updates_per_s": cell_updates / wall,
            "autotuned": {"cluster": cfg[0], "threads": cfg[1], "ctas_per_sm": cfg[2]}, "steps_max": max(steps),
            "l1_vs_cpu": per_nx, "cpu_baseline": cpu}


# --------------------------------------------------------------- accuracy

def _interior(a):
    return a[..., 3:-3, 3:-3, 3:-3]


def _advance_logged(step_fn, t, t_out, ke_fn, log):
    """time_advance's dt schedule one step at a time (maincycle.cpp:18-56), logging (t, KE)."""
    while abs(t_out - t) > 1e-12:
        t_new = step_fn(t, t_out)
        if t_new == t:
            break
        t = t_new
        log.append((t, ke_fn()))
    return t


def _ref_series(args):
    """Reference CPU run (oracle/_ref) of the isotropic workload to t_outs (spawned process)."""
    n, t_outs, interp, riemann = args
    sys.path.insert(0, ROOT)
    import math
    from ns3d_wcns_b200 import analysis
    from ns3d_wcns_b200.config import make_params
    from ns3d_wcns_b200.initial import isotropic_state
    from oracle import oracle
    P, G = make_params(n=(n, n, n), L=(2 * math.pi,) * 3, Ma=0.3, Re=400.0, Pr=0.72, cfl=0.5, dt_fixed=-1.0,
                       interpolation=interp, riemann=riemann, S_ref=110.4 / 273.15)
    s = oracle.RefSolver(P, G) if oracle.ref_available() else oracle.PortSolver(P, G)
    s.set_interior_prims(*isotropic_state((n, n, n), 1.4, 0.3, seed=0))

    def step(t, t_out):
        dt = s.timestep()
        if t + dt > t_out:
            dt = t_out - t
        if dt <= 1e-12:
            return t
        s.rk3_step(dt)
        return t + dt

    log, stats, t = [], {}, 0.0
    dV = (2 * math.pi / n) ** 3
    for t_out in t_outs:
        t = _advance_logged(step, t, t_out, s.total_energy, log)
        f = {k: _interior(s.get(k)) for k in ("rho", "u", "v", "w", "T")}
        st = analysis.turbulence_stats(f["rho"], f["u"], f["v"], f["w"], f["T"], 1.0 / 400.0, 110.4 / 273.15, dV)
        stats[t_out] = {"total_energy": st["total_energy"], "dissipation": st["dissipation"]}
    return {"log": log, "stats": stats, "kind": "reference" if oracle.ref_available() else "port"}


def accuracy_report(device: int, sizes=(256,), t_outs=(0.5, 1.0), ref_n: int = 0, series_dt: float = 0.1):
    """Mixed FP32/FP64 path against the plain FP64 path (itself pinned to the oracle at <= 1e-10
    over 10 steps) on the isotropic workload: relative L2 error of rho, u, v, w, E and of the
    spectrum E(k), k = 1..N/3, relative error of the kinetic energy and of the dissipation
    2 nu sum k^2 E(k) at each output time.  With ref_n > 0 also the time series of kinetic
    energy and dissipation of both GPU paths against the reference CPU run at ref_n^3."""
    import math
    import multiprocessing as mp
    import numpy as np
    import torch
    from ns3d_wcns_b200 import analysis
    from ns3d_wcns_b200.initial import isotropic_state
    from ns3d_wcns_b200.solver import Solver
    out = {}
    pool, fut = None, None
    if ref_n:
        outs = [round(series_dt * (i + 1), 10) for i in range(int(round(max(t_outs) / series_dt)))]
        pool = mp.get_context("spawn").Pool(1)
        fut = pool.apply_async(_ref_series, ((ref_n, outs, 3, 2),))
    fdev = f"cuda:{device}"
    mu0, S = 1.0 / 400.0, 110.4 / 273.15

    def run(n, precision, outs, keep):
        P, G = bench_params(n, precision)
        dV = (2 * math.pi / n) ** 3
        s = Solver(P, G, device=device)
        s.set_interior_primitives(*isotropic_state((n, n, n), 1.4, 0.3, seed=0))
        log, snaps, t, steps = [], {}, 0.0, 0
        t0 = time.perf_counter()

        def step(t, t_out):
            return s.time_advance(t_out, 1, t)[0]

        for t_out in outs:
            t = _advance_logged(step, t, t_out, s.total_energy, log)
            W = _interior(s.primitives())
            E = _interior(s.conserved()[4]) if keep is not None else None
            T = _interior(s.temperature())
            st = analysis.turbulence_stats(W[0], W[1], W[2], W[3], T, mu0, S, dV, device=fdev)
            snap = {"stats": st}
            if keep is not None:
                snap["fields"] = {"rho": W[0], "u": W[1], "v": W[2], "w": W[3], "E": E}
            snaps[t_out] = snap
            del W, T, E
        s.close()
        return {"log": log, "snaps": snaps, "wall_s": time.perf_counter() - t0}

    for n in sizes:
        ref = run(n, 0, t_outs, keep=True)
        mix = run(n, 1, t_outs, keep=True)
        rows = {}
        for t_out in t_outs:
            a, b = mix["snaps"][t_out], ref["snaps"][t_out]
            k = slice(1, n // 3 + 1)
            rows[str(t_out)] = {
                **{f"l2_{q}": analysis.rel_l2(a["fields"][q], b["fields"][q]) for q in ("rho", "u", "v", "w", "E")},
                "l2_spectrum_k1_N3": analysis.rel_l2(a["stats"]["spectrum"][k], b["stats"]["spectrum"][k]),
                "rel_total_energy": abs(a["stats"]["total_energy"] / b["stats"]["total_energy"] - 1),
                "rel_dissipation": abs(a["stats"]["dissipation"] / b["stats"]["dissipation"] - 1),
                "fp64_total_energy": b["stats"]["total_energy"], "fp64_dissipation": b["stats"]["dissipation"],
            }
        out[f"{n}^3"] = {"mixed_vs_fp64": rows, "steps_fp64": len(ref["log"]), "steps_mixed": len(mix["log"]),
                         "wall_s_fp64": ref["wall_s"], "wall_s_mixed": mix["wall_s"]}
        del ref, mix
        torch.cuda.empty_cache()

    if ref_n:
        outs = [round(series_dt * (i + 1), 10) for i in range(int(round(max(t_outs) / series_dt)))]
        gpu = {p: run(ref_n, p, outs, keep=None) for p in (0, 1)}
        r = fut.get()
        pool.close()
        series = []
        for t_out in outs:
            row = {"t": t_out, "ref_total_energy": r["stats"][t_out]["total_energy"],
                   "ref_dissipation": r["stats"][t_out]["dissipation"]}
            for p, name in ((0, "fp64"), (1, "mixed")):
                st = gpu[p]["snaps"][t_out]["stats"]
                row[f"{name}_rel_total_energy"] = abs(st["total_energy"] / row["ref_total_energy"] - 1)
                row[f"{name}_rel_dissipation"] = abs(st["dissipation"] / row["ref_dissipation"] - 1)
            series.append(row)
        # per-step kinetic energy along the whole run (same dt schedule when the steps agree)
        steps = min(len(r["log"]), len(gpu[0]["log"]))
        ke_fp64 = max(abs(gpu[0]["log"][i][1] / r["log"][i][1] - 1) for i in range(steps))
        out[f"reference_{ref_n}^3"] = {"kind": r["kind"], "series": series, "steps_ref": len(r["log"]),
                                       "steps_fp64": len(gpu[0]["log"]), "steps_mixed": len(gpu[1]["log"]),
                                       "max_rel_ke_fp64_per_step": ke_fp64}
    return out


# --------------------------------------------------------------- multi-GPU

def run_slabs(args, rank, world, local, dist):
    """N > 1: one 256^3 domain decomposed into N z-slabs (strong scaling), six
    halo planes of primitives and temperature exchanged with NCCL
    point-to-point operations after every RK stage, the CFL time step one
    MIN all-reduce per step (ns3d_wcns_b200/slab.py).  Device-timed, max over
    ranks; e2e adds each rank's upload of its slab from host memory at the
    start and the download of its owned planes at the end."""
    import numpy as np
    import torch
    from ns3d_wcns_b200.initial import isotropic_state
    from ns3d_wcns_b200.slab import SlabSolver, slab_plan
    n = args.n
    P, G = bench_params(n, 0)
    plan = slab_plan(n, world, rank, periodic=True)
    st = isotropic_state((n, n, n), 1.4, 0.3, seed=0)  # one global field, every rank takes its planes
    sv = SlabSolver(P, G, plan, device=local)
    stream = sv.stream  # the handle's kernels, the halo exchange and the events share it
    local_st = [np.ascontiguousarray(sv.local_block(f)) for f in st]
    del st
    sv.s.set_interior_primitives(*local_st)

    def steps(k):
        for _ in range(k):
            sv.rk3_step(sv.compute_timestep())

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    steps(args.warmup)
    dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sv.launch_count = 0
    clk.begin()
    e0.record(stream)
    steps(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk.end()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clocks = clk.stop()
    launches = sv.launch_count
    ke = sv.total_energy()
    dist.barrier()
    cells = float(n) ** 3
    value = cells * args.steps / (ms * 1e-3)

    e2e = None
    if not args.no_e2e:
        host = [torch.from_numpy(a).pin_memory().numpy() for a in local_st]
        out = torch.empty((5,) + sv.s.shape, dtype=torch.float64, pin_memory=True).numpy()

        def resident(k):
            sv.s.set_interior_primitives(*host)
            steps(k)
            sv.s._check(sv.s.lib.ns3d_download(sv.s.h, 0, sv.s._ptrs([out[q] for q in range(5)])))

        resident(args.warmup)
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        resident(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        mse = max_over_ranks(e0.elapsed_time(e1))
        nb_in = sum(a.nbytes for a in host)
        e2e = {"value": cells * args.steps / (mse * 1e-3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": world * nb_in / args.steps,
               "d2h_bytes_per_step": world * (out.nbytes + 8 * args.steps) / args.steps,
               "over_device_timed": (cells * args.steps / (mse * 1e-3)) / value,
               "path": "per rank: ns3d_set_interior_primitives of its slab, per step ns3d_compute_timestep + "
                       "MIN all-reduce + 3 x (ns3d_rk3_stage + NCCL halo exchange), ns3d_download at the end"}
    sv.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (one seeded isotropic field, decomposed)",
            "config": {"workload": WORKLOAD, "grid": [n, n, n],
                       "parallelism": f"z-slabs x{world}: {plan.owned}-{plan.owned + 1} owned planes a rank, "
                                      "6-plane halos exchanged by NCCL P2P after every RK stage",
                       "l2": "inputs larger than L2"},
            "e2e": e2e, "clocks": clocks, "gpu_launches": launches, "kinetic_energy_end": ke,
        }
        print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-512", action="store_true")
    ap.add_argument("--batch-problems", type=int, default=512)
    ap.add_argument("--batched-check", action="store_true",
                    help="batched report only, checking every Nx=200 problem and 8 of each larger Nx")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many host-loop RK3 steps of the workload at --n (plain FP64, or the mixed "
                         "path with --no-fp64) and exit: the case for one-kernel profiler captures")
    ap.add_argument("--no-fp64", action="store_true", help="with --profile-steps: the mixed path")
    ap.add_argument("--batch-profile", type=int, default=0,
                    help="run the first --batch-problems shock tubes of the batched benchmark for this many "
                         "steps (wavefront schedule, no checks) and exit: the case for profiler captures")
    ap.add_argument("--accuracy", default="", help="comma-separated grid sizes: accuracy report only")
    ap.add_argument("--accuracy-ref", type=int, default=0, help="also the reference CPU time series at this size")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference" or os.environ.get("NS3D_BENCH_ALLOW_SHORT"), \
        "at least 3 warm-up steps"

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.batched_check:
        import torch
        torch.cuda.set_device(local)
        rep = batched_report(local, args.batch_problems,
                             check=((200, 10 ** 6, "port"), (400, 8, "port"), (800, 8, "port"), (1600, 8, "port"),
                                    (200, 8, "reference")))
        print(json.dumps({"batched": rep}))
        return
    if args.batch_profile:
        import math
        import torch
        from ns3d_wcns_b200.batch import Batch, shock_tube_problems
        from ns3d_wcns_b200.config import make_params
        from ns3d_wcns_b200.initial import shock_tube_state
        torch.cuda.set_device(local)
        P, _ = make_params(n=(8, 4, 4), Ma=1.0, Re=math.inf, cfl=0.5, dt_fixed=-1.0, interpolation=0, riemann=0,
                           bcs=(3, 3, 0, 0, 0, 0))
        grids, left, right, t_end = shock_tube_problems(args.batch_problems, seed=5)
        with Batch(P, grids, t_end, device=local) as b:
            for i, g in enumerate(grids):
                b.set_interior_primitives(i, *shock_tube_state(g.global_nx, 4, 4, left[i], right[i]))
            b.set_config(0, 256, 1)
            b.run(args.batch_profile)
        print(json.dumps({"batch_profile": args.batch_profile, "problems": args.batch_problems}))
        return
    if args.profile_steps:
        import torch
        from ns3d_wcns_b200.initial import isotropic_state
        from ns3d_wcns_b200.solver import Solver
        torch.cuda.set_device(local)
        P, G = bench_params(args.n, 1 if args.no_fp64 else 0)
        with Solver(P, G, device=local) as s:
            stream = torch.cuda.Stream()
            s.set_stream(stream.cuda_stream)
            s.set_interior_primitives(*isotropic_state((args.n,) * 3, 1.4, 0.3, seed=0))
            for _ in range(args.profile_steps):
                s.rk3_step(s.compute_timestep())
            s.synchronize()
        print(json.dumps({"profile_steps": args.profile_steps, "n": args.n, "mixed": bool(args.no_fp64)}))
        return
    if args.accuracy:
        rep = accuracy_report(local, sizes=[int(x) for x in args.accuracy.split(",")], ref_n=args.accuracy_ref)
        print(json.dumps({"accuracy": rep}))
        return

    import numpy as np
    import torch
    from ns3d_wcns_b200 import _lib
    from ns3d_wcns_b200.initial import isotropic_state
    from ns3d_wcns_b200.solver import Solver

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if world > 1:
        try:
            run_slabs(args, rank, world, local, dist)
        finally:
            dist.destroy_process_group()
        return

    n = args.n
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()

    st = isotropic_state((n, n, n), 1.4, 0.3, seed=rank)
    # an explicit stream: the handles launch on it and the events are recorded on it
    # (ns3d_set_stream with the default stream's NULL would give a handle a private stream)
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_run(precision, profile):
        """K steps of the production time loop (ns3d_time_advance: CFL dt + RK3
        step with the dt schedule on the device, CUDA graphs), device-timed;
        then, outside the timed region, a short profiled pass for the
        per-kernel split (event profiling runs the host loop)."""
        P, G = bench_params(n, precision)
        s = Solver(P, G, device=local)
        s.set_stream(stream.cuda_stream)
        s.set_interior_primitives(*st)
        t_far = 1e30  # no clipping: every step takes its CFL dt
        t, _ = s.time_advance(t_far, args.warmup, 0.0)  # warm-up (captures the step graphs)
        barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.begin()
        e0.record(stream)
        t, done = s.time_advance(t_far, args.steps, t)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.end()
        ms = e0.elapsed_time(e1)
        clocks = clk.stop()
        launches = s.launches()
        assert done == args.steps
        barrier()
        prof = None
        if profile:
            # the same number of steps again, event-profiled per kernel (host loop)
            s.profile(True)
            for _ in range(args.steps):
                s.rk3_step(s.compute_timestep())
            prof = s.profile_report()
            s.profile(False)
        ke = s.total_energy()
        s.close()
        return max_over_ranks(ms), launches, prof, clocks, ke

    ms64, launches, prof, clocks, ke64 = timed_run(0, profile=True)
    cells = float(n) ** 3
    value = world * cells * args.steps / (ms64 * 1e-3)

    mixed = None
    if not args.no_mixed:
        msm, _, profm, _, kem = timed_run(1, profile=True)
        mixed = {"value": world * cells * args.steps / (msm * 1e-3), "unit": "cell-updates/s",
                 "ms_per_step": msm / args.steps, "over_fp64": ms64 / msm,
                 "kernels_ms": {k: round(v["ms"] / max(v["launches"], 1), 4) for k, v in (profm or {}).items()}}

    # roofline of the dominant kernel (algorithmic bytes per launch / event time)
    # sweep_z_stage (FP64: z-sweep with the RK update fused in): z-sweep 120 + stage 160
    # of the per-kernel figures, less the RHS write, its re-read and the stage's state read
    algo_bytes_per_cell = {"sweep_x": 80, "sweep_y": 120, "sweep_z": 120, "sweep_z_stage": 160,
                           "viscous_flux": 40 + 72,
                           "viscous_div": 72 + 64, "stage": 160, "cfl_dt": 40}
    dom = max(prof, key=lambda k: prof[k]["ms"])
    avg_ms = prof[dom]["ms"] / prof[dom]["launches"]
    achieved = algo_bytes_per_cell.get(dom, 0) * cells / (avg_ms * 1e-3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"traffic_{n}.txt")
    if os.path.exists(tpath):
        for ln in open(tpath):
            f = ln.split()
            if len(f) == 2 and not ln.startswith("#") and f[0] == dom:
                traffic = float(f[1])

    # FP64 pipe of the dominant kernel: its FP64 thread instructions per cell
    # (one-launch ncu capture, profiles/fp64_instr_per_cell_192.txt) over the
    # event time, against 64 FP64 lanes per SM per clock at the sampled clock
    fp64_pipe = None
    fpath = os.path.join(ROOT, "profiles", "fp64_instr_per_cell_192.txt")
    if os.path.exists(fpath):
        for ln in open(fpath):
            f = ln.split("#")[0].split()
            if len(f) == 2 and f[0] == dom:
                sms = torch.cuda.get_device_properties(local).multi_processor_count
                mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
                rate = float(f[1]) * cells / (avg_ms * 1e-3)
                peak64 = sms * 64 * mhz * 1e6
                fp64_pipe = {"achieved": rate, "peak": peak64, "unit": "FP64 thread-instructions/s",
                             "frac": rate / peak64, "fp64_instr_per_cell": float(f[1]),
                             "source": "profiles/fp64_instr_per_cell_192.txt (one-kernel ncu captures at 192^3)"}

    # end to end through the C ABI with host buffers (pinned)
    e2e = e2e_full = None
    if not args.no_e2e:
        P, G = bench_params(n, 0)
        s = Solver(P, G, device=local)
        s.set_stream(stream.cuda_stream)
        s.set_interior_primitives(*st)
        host = torch.empty((5, n + 6, n + 6, n + 6), dtype=torch.float64, pin_memory=True).numpy()
        host[...] = s.primitives()
        nbytes = 5 * (n + 6) ** 3 * 8
        monitor = 10

        def resident(k):
            """The drop-in's time_advance: upload once, per step the CFL dt and an RK3
            step, the monitor every 10th step and at step 1, download at the end."""
            s.upload_primitives(host)
            reads = 0
            for step in range(1, k + 1):
                s.rk3_step(s.compute_timestep())
                reads += 8
                if step % monitor == 0 or step == 1:
                    s.residuals()
                    s.total_energy()
                    reads += 48
            s._check(s.lib.ns3d_download(s.h, _lib.NS3D_PRIMITIVE, s._ptrs([host[q] for q in range(5)])))
            return reads

        def full_state(k):
            for _ in range(k):
                s.upload_primitives(host)
                s.rk3_step(s.compute_timestep())
                s._check(s.lib.ns3d_download(s.h, _lib.NS3D_PRIMITIVE, s._ptrs([host[q] for q in range(5)])))

        def timed(fn):
            fn(args.warmup)
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn(args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1))
            barrier()
            return ms, out

        mse, reads = timed(resident)
        e2e = {"value": world * cells * args.steps / (mse * 1e-3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": (nbytes + reads) / args.steps,
               "over_device_timed": None,
               "path": "ns3d_upload_primitives once; per step ns3d_compute_timestep + ns3d_rk3_step; "
                       "ns3d_residuals + ns3d_total_energy at step 1 and every 10th; ns3d_download at the end "
                       "(the drop-in's time_advance)"}
        msf, _ = timed(full_state)
        e2e_full = {"value": world * cells * args.steps / (msf * 1e-3), "unit": "cell-updates/s",
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 8,
                    "path": "per step ns3d_upload_primitives + ns3d_compute_timestep + ns3d_rk3_step + "
                            "ns3d_download"}
        s.close()

    if e2e is not None:
        e2e["over_device_timed"] = e2e["value"] / value

    # the mixed-precision config's larger grid: both paths at 512^3
    g512 = None
    if not args.no_512 and n == 256:
        st512 = isotropic_state((512, 512, 512), 1.4, 0.3, seed=rank)
        res = {}
        for prec, name in ((0, "fp64"), (1, "mixed")):
            P, G = bench_params(512, prec)
            s = Solver(P, G, device=local)
            s.set_stream(stream.cuda_stream)
            s.set_interior_primitives(*st512)
            t, _ = s.time_advance(1e30, args.warmup, 0.0)
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t, done = s.time_advance(1e30, args.steps, t)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1))
            s.close()
            res[name] = {"value": world * 512.0 ** 3 * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps}
        del st512
        torch.cuda.empty_cache()
        g512 = {**res, "mixed_over_fp64": res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"],
                "unit": "cell-updates/s", "steps": args.steps}

    adjoint = adjoint_hllc = adjoint_hyb = None
    if not args.no_adjoint and rank == 0:
        adjoint = adjoint_report(local)
        adjoint_hllc = adjoint_report(local, interp=2, riemann=2)
        adjoint_hyb = adjoint_report(local, interp=3, riemann=2, fd=False)
    batched = None
    if not args.no_batch and rank == 0:
        batched = batched_report(local, args.batch_problems)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms64 / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded isotropic field)",
            "config": {"workload": WORKLOAD, "grid": [n, n, n], "parallelism": "one GPU, whole domain",
                       "l2": "inputs larger than L2 (state 720 MB per copy)"},
            "e2e": e2e, "e2e_full_state": e2e_full, "mixed": mixed, "grid_512": g512,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "algorithmic_bytes_per_cell": algo_bytes_per_cell.get(dom), "fp64_pipe": fp64_pipe},
            "kernels_ms": {k: round(v["ms"] / max(v["launches"], 1), 4) for k, v in prof.items()},
            "kernels_ms_source": "CUDA events around each kernel, on the launching stream, in a pass of the same "
                                 "number of steps right after the timed region (the timed region runs the graph-"
                                 "captured device time loop, which event profiling cannot enter)",
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "kinetic_energy_end": ke64,
            "adjoint": adjoint, "adjoint_mdcd_linear_hllc": adjoint_hllc, "adjoint_benchmark_scheme": adjoint_hyb,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
