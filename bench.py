#!/usr/bin/env python
"""IMPES cell-steps/s on the B200 (mixed vs FP64 AMG-FGMRES at a 1e-6 residual).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 200x200x25 (1e6-cell) three-phase gas-injection case -- seeded
correlated log-normal permeability, 20-row black-oil PVT table, Stone II,
gravity, capillarity, 9 gas injectors at 2e5 sm3/d (entered as the equivalent
reservoir rate) and 16 BHP producers at 15 MPa, dt = 2 days.  A step is one full IMPES step (assembly,
Galerkin update of the frozen AMG hierarchy, FGMRES pressure solve to a 1e-6
Jacobi-scaled relative residual, explicit saturation update) with the state
resident in HBM; L2 is flushed (512 MiB write) before every timed step.

``value`` is the mixed-precision path (fp32 V-cycle in fp64 FGMRES); the same
protocol is applied to the all-fp64 path and reported under ``fp64``.  ``e2e``
repeats the measurement through the public ``Simulator.run_step`` with the state
copied from and back to pinned host memory inside the timed region.

Single grids do not shard: with N > 1 every rank runs its own replica (weak
scaling), timed on the device and reduced with max over ranks.

``--impl reference`` times the CPU restatement of the reference's own step (its
stand-alone V-cycle AMG with tol 1e-6 and 40 cycles) on the host cores, on a
bounded spatial sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(REPO, "oil-simulator-py_b200"), REPO):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "IMPES cell-steps/s, mixed vs FP64 AMG at 1e-6 residual; adjoint/forward time"
WORKLOAD = ("gas_injection_1m: 200x200x25 = 1,000,000 cells, ln k ~ N(ln 150 mD, 1.0^2) "
            "Gaussian-correlated (radius 5), 20-row black-oil PVT (Bo 1.3->1.1 with p), Stone II, "
            "gravity, capillarity, 9 gas injectors at 2e5 sm3/d given as reservoir rate "
            "(x Bg at 25 MPa) with global_rate_scale 0.05 and max_substeps 20 (the reference's "
            "million-cell settings), 16 BHP producers (15 MPa), dt 2 d")
WORKLOAD_SHORT = ("gas_injection_1m: 200x200x25 cells, correlated log-normal k, 20-row black-oil PVT, "
                  "Stone II, gravity, Pc, 9 gas injectors (2e5 sm3/d as reservoir rate, rate scale 0.05), "
                  "16 BHP producers, dt 2 d")
PRESSURE_TOL = 1e-6
L2_FLUSH_BYTES = 512 << 20
DEFAULT_P_MAX = 2               # interpolation row cap of the headline hierarchy
CPU_SAMPLE = (100, 100, 25)     # spatial sample of the workload for the CPU legs


def read_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------ CPU legs
def cpu_sample_workload(dims=CPU_SAMPLE, seed=2):
    from impes_b200 import scenarios
    nx, ny, nz = dims
    return scenarios.gas_injection_1m(seed=seed, nx=nx, ny=ny, nz=nz)


def reference_sample_dims(steps: int, warmup: int, full_steps: int = 8):
    """The spatial sample of the reference arm: CPU_SAMPLE while the run has at
    most `full_steps` steps, otherwise a laterally smaller piece (nz kept) whose
    steps take about as long in total, so a long --steps run still ends within
    a few minutes (a 100x100x25 step takes ~15 s on one core)."""
    total = max(steps, 0) + max(warmup, 1)
    if total <= full_steps:
        return CPU_SAMPLE
    scale = (full_steps / total) ** 0.5
    nx = max(32, int(round(CPU_SAMPLE[0] * scale)))
    ny = max(32, int(round(CPU_SAMPLE[1] * scale)))
    return (nx, ny, CPU_SAMPLE[2])


def _cpu_reference_worker(args):
    """One replica of the CPU sample (runs in a spawned process with one thread)."""
    steps, warmup, dims, seed, barrier = args
    for _p in (os.path.join(REPO, "oil-simulator-py_b200"), REPO):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    from oracle.amg import AMGSolver
    from oracle.impes import Model
    cfg, f = cpu_sample_workload(dims, seed=seed)
    m = Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"], pvt_table=f["pvt"])
    a = cfg["simulation"]["amg"]
    solver = AMGSolver(tol=1e-6, max_cycles=40, theta=a["theta"], max_levels=a["max_levels"],
                       coarsest_size=a["coarsest_size"], seed=0)
    dt = 2 * 86400.0
    for _ in range(max(warmup, 1)):       # the first step builds the hierarchy
        m.step(dt, solve=solver)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        m.step(dt, solve=solver)
    return m.N, time.perf_counter() - t0


def cpu_workers() -> int:
    """Host cores used by the CPU legs: every core this process may run on, up to
    16 (each replica holds its own AMG hierarchy, ~1 GB for the 100x100x25 sample)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(16, n))


def run_cpu_reference(steps: int, warmup: int, dims=CPU_SAMPLE):
    """The oracle's restatement of the reference step on the host cores: one
    replica of a `dims` spatial sample of the workload per core (scipy's sparse
    kernels are single-threaded, so the cores are used the way the GPU arm uses
    GPUs: independent replicas), timed from a common start.
    Returns (cell-steps/s over all replicas, seconds, cells per replica, cores,
    description)."""
    import multiprocessing as mp
    workers = cpu_workers()
    env_threads = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in env_threads:
        os.environ[k] = "1"
    try:
        if workers == 1:
            results = [_cpu_reference_worker((steps, warmup, dims, 2, None))]
        else:
            ctx = mp.get_context("spawn")
            with ctx.Manager() as mgr:
                bar = mgr.Barrier(workers)
                with ctx.Pool(workers) as pool:
                    results = pool.map(_cpu_reference_worker,
                                       [(steps, warmup, dims, 2, bar) for _ in range(workers)])
    finally:
        for k, v in env_threads.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    cells = results[0][0]
    secs = max(r[1] for r in results)
    desc = (f"oracle restatement of the reference IMPES step (stand-alone RS-AMG V-cycles, tol 1e-6 "
            f"equilibrated, max 40 cycles) on a {dims[0]}x{dims[1]}x{dims[2]} sample of the "
            f"workload, {workers} replicas (one per core, one thread each), {steps} timed steps after "
            f"{max(warmup, 1)} warm-up (setup excluded)")
    return workers * cells * steps / secs, secs, cells, workers, desc


# ------------------------------------------------------------------ GPU legs
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 200 ms while the timed
    region runs; the raw samples go to `directory` (a temporary one by default)."""

    def __init__(self, index: int, directory: str | None = None):
        import tempfile
        self.index = index
        self.proc = None
        self.path = os.path.join(directory or tempfile.gettempdir(), f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx = float(parts[1])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[3:7]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def make_sim(cfg, fields, precision, device, restart=30, solver="gmres_amg", warm_start="extrapolate",
             trunc=0, smoother="l1jacobi", tol=PRESSURE_TOL, light=0):
    """FGMRES + V-cycle (solver="gmres_amg"), or the plain stand-alone V-cycles of
    the reference (solver="amg"), both stopping at PRESSURE_TOL in the Jacobi norm;
    `trunc` caps the interpolation's row length (0: the reference's interpolation);
    levels of at most `light` rows smooth once before and once after their coarse
    correction (0: three and two sweeps on every level, as the reference)."""
    from impes_b200.simulator import build_from_config
    c = json.loads(json.dumps(cfg))
    c["simulation"]["pressure_solver"] = solver
    c["simulation"]["amg"].update({"tol": tol, "norm": "jacobi", "precision": precision,
                                   "restart": restart, "max_iters": 600, "max_cycles": 3000, "seed": 0,
                                   "warm_start": warm_start, "p_max_elements": int(trunc),
                                   "smoother": smoother, "light_sweep_rows": int(light)})
    return build_from_config(c, fields, device=device)


def time_steps(sim, steps, dt, flush, stream, nvtx_last=False):
    """Device time of `steps` IMPES steps (L2 flushed before each, outside the
    events).  With nvtx_last the last step runs inside an NVTX range named
    "impes_step", which a profiler can select (ncu --nvtx --nvtx-include)."""
    import torch
    total = 0.0
    iters = []
    for q in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        mark = nvtx_last and q == steps - 1
        if mark:
            torch.cuda.nvtx.range_push("impes_step")
        a.record(stream)
        ok = sim.run_step(dt)
        b.record(stream)
        if mark:
            torch.cuda.nvtx.range_pop()
        b.synchronize()
        if not ok:
            raise RuntimeError("IMPES step failed to converge")
        total += a.elapsed_time(b)
        iters.append(sim.last_krylov["iterations"])
    return total, iters


def time_e2e(sim, fl, steps, dt, flush, stream):
    """Public API with host state: H2D of (p, Sw, Sg), run_step, D2H of (p, Sw, Sg)."""
    import torch
    host = [t.detach().cpu().pin_memory() for t in (fl.pressure, fl.s_w, fl.s_g)]
    total = 0.0
    iters = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fl.pressure.copy_(host[0], non_blocking=True)
        fl.s_w.copy_(host[1], non_blocking=True)
        fl.s_g.copy_(host[2], non_blocking=True)
        if not sim.run_step(dt):
            raise RuntimeError("IMPES step failed to converge")
        host[0].copy_(fl.pressure, non_blocking=True)
        host[1].copy_(fl.s_w, non_blocking=True)
        host[2].copy_(fl.s_g, non_blocking=True)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
        iters.append(sim.last_krylov["iterations"])
    nbytes = sum(h.numel() * h.element_size() for h in host)
    return total, nbytes, iters


def total_mass(fl, pv):
    """Mass in place, sum of PV * S * rho(p) over the phases (kg), as the
    reference's mass-balance test forms it (tests/test_impes_3phase.py:16-30)."""
    return float((pv * (fl.s_w * fl.rho_w + fl.s_o * fl.rho_o + fl.s_g * fl.rho_g)).sum())


def net_inflow(sim):
    """Cumulative net mass inflow (kg) of the run, sim.mass_balance (in - out)
    summed over the phases (simulation.py:1511-1525)."""
    mb = sim.mass_balance
    return sum(mb[ph]["in"] - mb[ph]["out"] for ph in ("water", "oil", "gas"))


def read_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(REPO, "profiles", f"{kernel}_gas_injection_1m.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


ADJOINT_WORKLOAD = ("adjoint_case: 64x64x8 oil-water, ln k ~ N(ln 100 mD, 0.7^2), 50 steps of 2 d, "
                    "J = sum (q_o - q_target)^2 at the producer (flux-balance rate), targets from a "
                    "second seeded k field, gradient w.r.t. ln k and porosity, checkpoints every 10 steps, "
                    "FGMRES to 1e-10 (Jacobi norm) in the forward and adjoint solves")


def run_adjoint(device):
    """Forward run and adjoint gradient of the history-matching objective; device
    times come from the library's own CUDA events (forward run; reverse sweep
    with the recomputation of the checkpointed segments)."""
    import torch
    from impes_b200 import scenarios
    from impes_b200.adjoint import misfit_gradient, producer_rates
    steps = 50
    cfg, f = scenarios.adjoint_case(seed=3, steps=steps)
    _, f2 = scenarios.adjoint_case(seed=5, steps=steps)
    dt = cfg["simulation"]["time_step_days"] * 86400.0
    target = producer_rates(cfg, dict(f2, poro=f["poro"]), steps, dt, tol=1e-10, device=device)
    runs = []
    for _ in range(3):          # the first call is a warm-up
        out = misfit_gradient(cfg, f, target, steps, dt, checkpoint_every=10, tol=1e-10,
                              adjoint_tol=1e-10, device=device)
        runs.append(out["stats"])
    st = runs[-1]
    # the same gradient with the fp32 V-cycle inside both FGMRES solves, against
    # the fp64 one (norm-relative)
    mixed = misfit_gradient(cfg, f, target, steps, dt, checkpoint_every=10, tol=1e-10, adjoint_tol=1e-10,
                            device=device, precision="mixed")
    g64 = torch.cat([out["g_lnk"].reshape(-1), out["g_poro"].reshape(-1)])
    g32 = torch.cat([mixed["g_lnk"].reshape(-1), mixed["g_poro"].reshape(-1)])
    mixed_err = float((g32 - g64).norm() / g64.norm())
    fwd = statistics.median(r["forward_ms"] for r in runs[1:])
    rev = statistics.median(r["reverse_ms"] for r in runs[1:])
    return {"workload": ADJOINT_WORKLOAD, "cells": 64 * 64 * 8, "steps": steps,
            "forward_ms": fwd, "reverse_ms": rev, "adjoint_over_forward": rev / fwd,
            "gradient_over_forward": (fwd + rev) / fwd, "J": st["J"],
            "forward_fgmres_iterations": st["forward_iterations"],
            "adjoint_fgmres_iterations": st["adjoint_iterations"],
            "recomputed_steps": st["recomputed_steps"],
            "mixed_precision_gradient_rel_err_vs_fp64": mixed_err,
            "mixed_forward_ms": mixed["stats"]["forward_ms"], "mixed_reverse_ms": mixed["stats"]["reverse_ms"]}


ENSEMBLE_WORKLOAD = ("ensemble: 64 oil-water realisations (seed 4), nx, ny in {32,48,64,96,128}, "
                     "nz in {4,8,16}, sigma_lnk in [0.3, 1.2], corner wells, 30 steps of 1 d each, "
                     "FGMRES(60) + fp32 V-cycle to 1e-6 (Jacobi norm); one hierarchy per member, "
                     "P capped at 2/row, one sweep before/after on levels of <= 30% of the member's cells; "
                     "members sharded across ranks by cell count")


def run_ensemble(device, rank, world, dist, steps=30, workers=8, warmup=3, loop_steps=3, trunc=DEFAULT_P_MAX,
                 light_frac=0.3):
    """All members advanced `steps` steps after `warmup` untimed ones; the time is
    the device span of the library's run (max over ranks).  The warm-up builds
    every member's hierarchy and reaches the paths the first step does not (the
    time-extrapolated iterate and its kernels, further V-cycle graphs): after a
    single warm-up step the first timed run took 4.5-6.0 s, after three 3.9 s,
    and later runs 3.1-3.4 s.

    Beside it: the same members looped one at a time through the single-instance
    path (Simulator.run_step per member per step, as the reference's callers do,
    simulation.py:126-135, rl_env.py:90-108) for `loop_steps` steps, and the
    mixed-precision members' final states against an all-fp64 run of the same
    members and steps.

    Every member's hierarchy is the headline's kind: interpolation capped at
    `trunc` entries per row, one sweep before and one after the coarse
    correction on the levels of at most `light_frac` of the member's cells
    (trunc 0 and light_frac 0: the reference's hierarchy and cycle)."""
    import torch
    from impes_b200 import scenarios
    from impes_b200.ensemble import Ensemble, gather
    cases = scenarios.ensemble(seed=4, members=64, steps=steps)
    for cfg, _ in cases:
        nx, ny, nz = cfg["reservoir"]["dimensions"]
        am = cfg["simulation"].setdefault("amg", {})
        am["p_max_elements"] = int(trunc)
        am["light_sweep_rows"] = int(light_frac * nx * ny * nz) if trunc else 0
    dt = cases[0][0]["simulation"]["time_step_days"] * 86400.0
    amg = {"tol": PRESSURE_TOL, "norm": "jacobi", "precision": "mixed", "restart": 60, "max_iters": 1000}
    ens = Ensemble(cases, device=device, rank=rank, world=world, workers=workers, amg=amg)
    ens.run(max(1, warmup), dt)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    ens.run(steps, dt)
    t = torch.tensor([ens.last_span_ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    summ = gather(ens.summary(), world)
    final = [(s.fluid.pressure.clone(), s.fluid.s_w.clone(), s.fluid.s_g.clone()) for s in ens.sims]
    # the single-instance loop, on the same members (their trajectories go on)
    stream = torch.cuda.current_stream(device)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(loop_steps):
        for sim in ens.sims:
            if not sim.run_step(dt):
                raise RuntimeError("ensemble member failed to converge in the loop baseline")
    b.record(stream)
    b.synchronize()
    tl = torch.tensor([a.elapsed_time(b)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(tl, op=dist.ReduceOp.MAX)
    ens.close()
    # all-fp64 run of the same members and steps
    ens64 = Ensemble(cases, device=device, rank=rank, world=world, workers=workers,
                     amg=dict(amg, precision="fp64"))
    ens64.run(max(1, warmup), dt)
    ens64.run(steps, dt)
    ds, dp = 0.0, 0.0
    for (p, sw, sg), s64 in zip(final, ens64.sims):
        fl = s64.fluid
        ds = max(ds, float((sw - fl.s_w).abs().max()), float((sg - fl.s_g).abs().max()))
        dp = max(dp, float((p - fl.pressure).abs().max() / fl.pressure.abs().max()))
    ens64.close()
    drift = torch.tensor([ds, dp], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(drift, op=dist.ReduceOp.MAX)
    total = sum(ens.cells)
    ms = float(t.item())
    loop_cs = total * loop_steps / (float(tl.item()) / 1e3)
    cs = total * steps / (ms / 1e3)
    return {"workload": ENSEMBLE_WORKLOAD, "members": len(ens.cells), "cells": total, "steps": steps,
            "ms": ms, "cell_steps_per_s": cs, "workers_per_gpu": workers,
            "warmup_steps": max(1, warmup),
            "loop_steps": loop_steps, "loop_ms": float(tl.item()), "loop_cell_steps_per_s": loop_cs,
            "speedup_vs_loop": cs / loop_cs,
            "drift_s_abs_vs_fp64": float(drift[0]), "drift_p_rel_vs_fp64": float(drift[1]),
            "fgmres_iterations": int(sum(s["iterations"] for s in summ)),
            "all_converged": all(s["status"] == 0 for s in summ), "scaling": "strong"}


def sig(x, n=4):
    """x rounded to n significant digits (floats), for the compact result line."""
    if x is None or isinstance(x, (bool, int, str)):
        return x
    return float(f"{x:.{n}g}")


def run_variant(args, cfg, fields, precision, device, dt, flush, stream, dist, rank, local, trunc,
                label):
    """Setup + W warm-up steps, K device-timed steps (headline protocol), K steps
    with the library's phase timers, K steps end to end through run_step with
    host state.  Returns the measurements of this (precision, interpolation)."""
    import torch
    from impes_b200 import _lib
    _, fl, _, sim = make_sim(cfg, fields, precision, device, restart=args.restart,
                             warm_start=False if args.warm_start == "zero" else args.warm_start,
                             trunc=trunc, smoother=args.smoother, light=args.light_sweep_rows if trunc else 0)
    pv = sim.porous_volume.reshape(fl.s_w.shape)
    m0 = total_mass(fl, pv)
    torch.cuda.synchronize()
    t_setup = time.perf_counter()
    for _ in range(args.warmup):           # the first warm-up step builds the hierarchy
        if not sim.run_step(dt):
            raise RuntimeError("warm-up step failed to converge")
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.kernel_launches()
    with ClockSampler(local, args.clocks_dir) as clk:
        ms, iters = time_steps(sim, args.steps, dt, flush, stream, nvtx_last=args.nvtx)
    launches = _lib.kernel_launches() - launches0
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    tmax = torch.tensor([ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    # phase timers (CUDA events around every phase and every wide-level sweep,
    # recorded inside the V-cycle graphs) run on K further steps, kept out of the
    # headline region because their event records lengthen each V-cycle
    _lib.timing_enable(True)
    _lib.timing_collect()
    ms_inst, iters_inst = time_steps(sim, args.steps, dt, flush, stream)
    phases = _lib.timing_collect()
    _lib.timing_enable(False)
    e2e_ms, e2e_bytes, e2e_iters = time_e2e(sim, fl, args.steps, dt, flush, stream)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    levels = sim.amg_levels()
    level_us = sim.amg_profile_levels(precision, reps=20) if args.level_profile else None
    nnz = [lv[1] for lv in levels]
    oc = sum(nnz) / max(nnz[0], 1) if nnz else None
    m1 = total_mass(fl, pv)
    inflow = net_inflow(sim)
    if rank == 0:
        print(f"[bench] {label}: levels (n, nnz, nc, p_nnz, coarsest, columns) = {levels}", file=sys.stderr)
        print(f"[bench] {label}: phases {phases}", file=sys.stderr)
        if level_us is not None:
            print(f"[bench] {label}: per-level us (sweep, residual, restrict, prolong) = "
                  f"{[tuple(round(v, 2) for v in t) for t in level_us]}", file=sys.stderr)
    out = dict(ms=float(tmax.item()), iters=iters, phases=phases, clocks=clk.summary(), ms_inst=ms_inst,
               iters_inst=iters_inst, launches=launches, e2e_ms=float(te.item()), e2e_bytes=e2e_bytes,
               e2e_iters=e2e_iters, setup_s=setup_s, p=fl.pressure.clone(), sw=fl.s_w.clone(),
               sg=fl.s_g.clone(), oc=oc, levels=len(levels),
               layout0=(levels[0][7][1 if precision == "mixed" else 0] if levels else None),
               mass_err=abs((m1 - m0) - inflow) / max(abs(m0), 1e-300),
               steps_run=args.warmup + 3 * args.steps,
               state={"sw": [float(fl.s_w.min()), float(fl.s_w.max())],
                      "sg": [float(fl.s_g.min()), float(fl.s_g.max())],
                      "p_MPa": [float(fl.pressure.min()) / 1e6, float(fl.pressure.max()) / 1e6]})
    sim.close()
    del sim, fl
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def run_ours(args, world, rank, local):
    import torch
    from impes_b200 import scenarios

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=device)
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.lower().split("x"))
        cfg, fields = scenarios.gas_injection_1m(seed=2, nx=nx, ny=ny, nz=nz)
    else:
        cfg, fields = scenarios.gas_injection_1m(seed=2)
    dt = cfg["simulation"]["time_step_days"] * 86400.0
    cells = cfg["reservoir"]["dimensions"][0] * cfg["reservoir"]["dimensions"][1] * cfg["reservoir"]["dimensions"][2]
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    if args.light_sweep_rows < 0:
        args.light_sweep_rows = int(0.3 * cells)

    # (precision, interpolation cap) variants; the headline is the mixed path on
    # the --p-max-elements hierarchy, and the reference's own interpolation (cap 0)
    # is measured beside it when the headline truncates
    trunc = args.p_max_elements
    variants = []
    precisions = ("fp64", "mixed") if args.precision == "both" else (args.precision,)
    for precision in precisions:
        variants.append((precision, trunc))
    if args.precision == "both" and trunc > 0 and not args.no_reference_hierarchy:
        variants += [("fp64", 0), ("mixed", 0)]
    results = {}
    for precision, tr in variants:
        label = f"{precision}/trunc{tr}"
        results[(precision, tr)] = run_variant(args, cfg, fields, precision, device, dt, flush, stream, dist,
                                               rank, local, tr, label)

    tight = None
    if args.precision == "both":
        # the same number of steps in fp64 solved to 1e-10: how far the 1e-6
        # solve tolerance alone moves the state (against the mixed-vs-fp64 drift)
        r64 = results[("fp64", trunc)]
        _, flt, _, simt = make_sim(cfg, fields, "fp64", device, restart=args.restart, trunc=trunc, tol=1e-10,
                                   light=args.light_sweep_rows)
        pvt_ = simt.porous_volume.reshape(flt.s_w.shape)
        m0t = total_mass(flt, pvt_)
        for _ in range(r64["steps_run"]):
            if not simt.run_step(dt):
                raise RuntimeError("tight fp64 step failed to converge")
        tight = {"s_abs": float(max((flt.s_w - r64["sw"]).abs().max(), (flt.s_g - r64["sg"]).abs().max())),
                 "p_rel": float((flt.pressure - r64["p"]).abs().max() / flt.pressure.abs().max()),
                 "steps": r64["steps_run"],
                 "mass_err": abs((total_mass(flt, pvt_) - m0t) - net_inflow(simt)) / max(abs(m0t), 1e-300)}
        # and the mixed path solved to 1e-10 over the same steps: the precision's
        # own share of the drift once the tolerance no longer dominates it
        _, flm, _, simm = make_sim(cfg, fields, "mixed", device, restart=args.restart, trunc=trunc, tol=1e-10,
                                   light=args.light_sweep_rows)
        for _ in range(r64["steps_run"]):
            if not simm.run_step(dt):
                raise RuntimeError("tight mixed step failed to converge")
        tight["mixed_s_abs"] = float(max((flm.s_w - flt.s_w).abs().max(), (flm.s_g - flt.s_g).abs().max()))
        tight["mixed_p_rel"] = float((flm.pressure - flt.pressure).abs().max() / flt.pressure.abs().max())
        simm.close()
        simt.close()
        del simt, flt, simm, flm
        torch.cuda.empty_cache()

    plain = None
    if args.precision == "both" and not args.no_plain:
        # the plain FP64 GPU path: the reference's stand-alone V-cycles on the
        # reference's hierarchy, fp64, to the same 1e-6 Jacobi-scaled residual
        # (fewer timed steps: it is slow)
        _, flp, _, simp = make_sim(cfg, fields, "fp64", device, solver="amg", trunc=0)
        for _ in range(args.warmup):
            simp.run_step(dt)
        psteps = max(1, min(args.steps, 3))
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ms_p, it_p = time_steps(simp, psteps, dt, flush, stream)
        tp = torch.tensor([ms_p], dtype=torch.float64, device=device)
        if dist is not None:
            dist.all_reduce(tp, op=dist.ReduceOp.MAX)
        plain = dict(ms=float(tp.item()), iters=it_p, steps=psteps)
        simp.close()
        del simp, flp
        torch.cuda.empty_cache()
    adjoint = None
    if args.precision == "both" and not args.no_adjoint and rank == 0:
        adjoint = run_adjoint(device)
    ensemble = None
    if args.precision == "both" and not args.no_ensemble:
        ensemble = run_ensemble(device, rank, world, dist, warmup=max(3, args.warmup),
                                loop_steps=args.ensemble_loop_steps)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    hbm_peak, peak_kind = read_peaks()
    steps = args.steps
    if args.precision != "both":
        r = results[(args.precision, trunc)]
        print(json.dumps({"precision": args.precision, "p_max_elements": trunc, "smoother": args.smoother,
                          "light_sweep_rows": args.light_sweep_rows,
                          "ms_per_step": r["ms"] / steps, "vcycles_per_step": statistics.mean(r["iters"]),
                          "operator_complexity": r["oc"], "levels": r["levels"],
                          "phases": r["phases"], "gpu_launches": r["launches"]}), flush=True)
        return
    mixed, fp64 = results[("mixed", trunc)], results[("fp64", trunc)]
    value = world * cells * steps / (mixed["ms"] / 1e3)
    fp64_value = world * cells * steps / (fp64["ms"] / 1e3)
    # dominant kernel: the l1-Jacobi sweep of the wide coarse levels (k_csr_stream
    # and k_csr_rows, Y_SMOOTH) when the hierarchy has such levels, else level 0's
    # sweeps: the grid-tile launches (two sweeps, and the residual before the
    # coarse correction) where level 0 is a grid's DIA, else the single sweep;
    # timed per launch by the library's CUDA events
    ph = mixed["phases"]
    key = "smooth_wide" if ph["smooth_wide"][0] else ("tile_l0" if ph.get("tile_l0", (0,))[0] else "smooth_l0")
    n_s, ms_s, by_s = mixed["phases"][key]
    achieved = by_s / (ms_s / 1e3) / 1e9
    traffic = read_traffic(key)
    share = {k: round(v[1] / mixed["ms_inst"], 4) for k, v in mixed["phases"].items() if k != "solve"}
    drift_sw = float(max((mixed["sw"] - fp64["sw"]).abs().max(), (mixed["sg"] - fp64["sg"]).abs().max()))
    drift_p = float((mixed["p"] - fp64["p"]).abs().max() / fp64["p"].abs().max())
    vps = statistics.mean(mixed["iters"])
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "cell-steps/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": mixed["ms"] / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 Krylov/assembly/saturation + f32 V-cycle",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": WORKLOAD_SHORT, "cells": cells, "precision": "mixed",
                   "solver": (f"FGMRES({args.restart}) + RS-AMG V-cycle, P capped at {trunc}/row, "
                              f"one sweep before/after on levels of <= {args.light_sweep_rows} rows")
                             if trunc else f"FGMRES({args.restart}) + RS-AMG V-cycle",
                   "tol": PRESSURE_TOL, "norm": "Jacobi-scaled", "l2": "flushed before each step",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"kernel": "wide-level l1-Jacobi sweep" if key == "smooth_wide"
                     else ("level-0 grid-tile l1-Jacobi sweeps (k_dia_tile: two sweeps, + residual "
                           "before the coarse correction), fp32" if key == "tile_l0"
                           else f"level-0 l1-Jacobi sweep, fp32, {str(mixed.get('layout0')).upper()} layout"),
                     "bound": "hbm", "achieved": sig(achieved), "peak": hbm_peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": sig(achieved / hbm_peak, 3), "traffic": traffic},
        "e2e": {"value": sig(world * cells * steps / (mixed["e2e_ms"] / 1e3)), "unit": "cell-steps/s",
                "h2d_bytes_per_step": mixed["e2e_bytes"], "d2h_bytes_per_step": mixed["e2e_bytes"],
                "vcycles_per_step": sig(statistics.mean(mixed["e2e_iters"]), 3)},
        "clocks": mixed["clocks"],
        "gpu_launches": mixed["launches"],
        "vcycles_per_step": sig(vps, 3),
        "operator_complexity": sig(mixed["oc"], 3),
        "fp64": {"value": sig(fp64_value), "ms_per_step": sig(fp64["ms"] / steps),
                 "vcycles_per_step": sig(statistics.mean(fp64["iters"]), 3),
                 "mixed_speedup": sig(fp64["ms"] / mixed["ms"], 3)},
        "drift_vs_fp64": {"s_abs": sig(drift_sw, 2), "p_rel": sig(drift_p, 2), "steps": mixed["steps_run"]},
        "mass_balance_error": {"mixed": sig(mixed["mass_err"], 2), "fp64": sig(fp64["mass_err"], 2),
                               "steps": mixed["steps_run"]},
    }
    if tight is not None:
        line["fp64_tol_1e-6_vs_1e-10"] = {"s_abs": sig(tight["s_abs"], 2), "p_rel": sig(tight["p_rel"], 2)}
        line["drift_vs_fp64_at_1e-10"] = {"s_abs": sig(tight["mixed_s_abs"], 2), "p_rel": sig(tight["mixed_p_rel"], 2),
                                          "steps": tight["steps"]}
        line["mass_balance_error"]["fp64_tol_1e-10"] = sig(tight["mass_err"], 2)
    if ("mixed", 0) in results and trunc:
        rm, rf = results[("mixed", 0)], results[("fp64", 0)]
        line["ref_interp"] = {"ms_mixed": sig(rm["ms"] / steps), "ms_fp64": sig(rf["ms"] / steps),
                              "vcycles_per_step": sig(statistics.mean(rm["iters"]), 3),
                              "operator_complexity": sig(rm["oc"], 3),
                              "mixed_speedup": sig(rf["ms"] / rm["ms"], 3)}
    if plain is not None:
        line["plain_fp64_vcycle"] = {"ms_per_step": sig(plain["ms"] / plain["steps"]),
                                     "vcycles_per_step": sig(statistics.mean(plain["iters"]), 3),
                                     "mixed_speedup": sig((plain["ms"] / plain["steps"]) / (mixed["ms"] / steps), 3)}
    if adjoint is not None:
        line["adjoint"] = {"forward_ms": sig(adjoint["forward_ms"]), "reverse_ms": sig(adjoint["reverse_ms"]),
                           "gradient_over_forward": sig(adjoint["gradient_over_forward"], 3),
                           "mixed_grad_err_vs_fp64": sig(adjoint["mixed_precision_gradient_rel_err_vs_fp64"], 2)}
    if ensemble is not None:
        line["ensemble"] = {k: sig(ensemble[k]) for k in ("cell_steps_per_s", "loop_cell_steps_per_s",
                                                          "speedup_vs_loop", "drift_s_abs_vs_fp64")
                            if k in ensemble}
    if not args.no_cpu_baseline and world == 1:
        v, secs, ccells, cores, desc = run_cpu_reference(steps=1, warmup=1)
        line["cpu_baseline"] = {"value": sig(v), "unit": "cell-steps/s", "cores": cores, "kind": "port",
                                "sample": f"oracle port, {CPU_SAMPLE[0]}x{CPU_SAMPLE[1]}x{CPU_SAMPLE[2]} x {cores} replicas"}
        cpu_detail = {"value": v, "seconds": secs, "cells_per_replica": ccells, "description": desc}
    else:
        cpu_detail = None
    detail = {
        "workload": WORKLOAD,
        "results": {f"{p}/trunc{t}": {k: v for k, v in r.items() if k not in ("p", "sw", "sg")}
                    for (p, t), r in results.items()},
        "phase_share_mixed": share,
        "roofline": {"bytes_per_launch": by_s / max(n_s, 1), "avg_launch_us": ms_s / max(n_s, 1) * 1e3,
                     "launches_timed": n_s,
                     "level0_sweep": {"GBs": mixed["phases"]["smooth_l0"][2] / max(mixed["phases"]["smooth_l0"][1], 1e-9) / 1e6,
                                      "launches": mixed["phases"]["smooth_l0"][0]},
                     "level0_tiles": {"GBs": ph["tile_l0"][2] / max(ph["tile_l0"][1], 1e-9) / 1e6,
                                      "launches": ph["tile_l0"][0]}},
        "plain_fp64_vcycle": plain, "adjoint": adjoint, "ensemble": ensemble, "cpu_baseline": cpu_detail,
    }
    print("[bench-detail] " + json.dumps(detail), file=sys.stderr, flush=True)
    if args.detail_out:
        with open(args.detail_out, "w") as f:
            json.dump(detail, f, indent=1)
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank, local):
    if rank != 0:
        return
    dims = reference_sample_dims(args.steps, args.warmup)
    v, secs, cells, cores, desc = run_cpu_reference(steps=args.steps, warmup=args.warmup, dims=dims)
    line = {
        "metric": METRIC, "impl": "reference", "value": v, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": WORKLOAD, "cells": cells, "sample": list(dims),
                   "pressure_solver": "stand-alone RS-AMG V-cycles (reference semantics)",
                   "pressure_tol": PRESSURE_TOL, "residual_norm": "||D^-1/2 r|| / ||D^-1/2 b||"},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clocks-dir", default=None,
                    help="directory for the raw nvidia-smi clock samples (default: a temporary one)")
    ap.add_argument("--restart", type=int, default=60, help="FGMRES restart length")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 V-cycle baseline")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-member ensemble measurement")
    ap.add_argument("--warm-start", default="extrapolate", choices=["extrapolate", "quadratic", "previous", "zero"],
                    help="FGMRES first iterate: extrapolated pressure, previous pressure, or zero")
    ap.add_argument("--grid", default=None,
                    help="NXxNYxNZ: a smaller grid of the same workload (profiling captures only)")
    ap.add_argument("--precision", choices=["both", "mixed", "fp64"], default="both",
                    help="both (the benchmark line) or one path only (profiling runs)")
    ap.add_argument("--p-max-elements", type=int, default=DEFAULT_P_MAX,
                    help="interpolation row cap of the benchmarked hierarchy (0: the reference's "
                         "interpolation)")
    ap.add_argument("--light-sweep-rows", type=int, default=-1,
                    help="levels of at most this many rows smooth once before and once after their "
                         "coarse correction (capped hierarchy only; 0: three and two sweeps everywhere; "
                         "default: 30%% of the cell count, every level below the first coarse one "
                         "on the 1e6-cell hierarchy)")
    ap.add_argument("--smoother", choices=["l1jacobi", "chebyshev"], default="l1jacobi",
                    help="V-cycle smoother of the benchmarked hierarchy")
    ap.add_argument("--no-reference-hierarchy", action="store_true",
                    help="skip the measurement on the reference's own interpolation")
    ap.add_argument("--ensemble-loop-steps", type=int, default=3,
                    help="steps of the loop-the-single-path ensemble baseline")
    ap.add_argument("--detail-out", default=None, help="write the detailed results as JSON here")
    ap.add_argument("--level-profile", action="store_true",
                    help="time each level's sweep, residual, restriction and prolongation (stderr)")
    ap.add_argument("--nvtx", action="store_true",
                    help="mark the last headline step with an NVTX range \"impes_step\" for profilers")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
