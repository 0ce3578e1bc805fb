"""Ensembles of independent realisations (no counterpart in the reference,
whose callers loop over ``Simulator.run_step`` one run at a time).

Each member is an ordinary ``Simulator`` (its own model, AMG hierarchy and
state), so its trajectory is exactly the single-run trajectory.  ``run``
advances all members with ``impes_ensemble_run``: a native thread pool, one CUDA
stream per worker, members taken largest first.

Across GPUs the members shard with no data-path collective: ``partition``
assigns them to ranks by cell count (greedy, largest first onto the least
loaded rank), each rank runs its share, and ``gather`` collects the per-member
summaries (``torch.distributed.all_gather_object``; gloo or NCCL).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .simulator import build_from_config

__all__ = ["partition", "Ensemble", "gather"]


def partition(cells: Sequence[int], world: int) -> list[list[int]]:
    """Member indices per rank: largest first onto the least loaded rank (ties to
    the lower rank), each rank's list in ascending member order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for m in sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(m)
        load[r] += int(cells[m])
    return [sorted(v) for v in out]


def gather(local: list[dict], world: int) -> list[dict]:
    """All members' summaries on every rank, ordered by member index."""
    if world > 1:
        import torch.distributed as dist
        parts: list = [None] * world
        dist.all_gather_object(parts, local)
        local = [s for part in parts for s in part]
    return sorted(local, key=lambda s: s["member"])


class Ensemble:
    """The members of ``cases`` (a list of (config, fields)) assigned to ``rank``."""

    def __init__(self, cases: Sequence[tuple], device="cuda", rank: int = 0, world: int = 1,
                 workers: int = 8, amg: Optional[dict] = None):
        self.device = torch.device(device)
        self.cells = [int(np.prod(c[0]["reservoir"]["dimensions"])) for c in cases]
        self.members = partition(self.cells, world)[rank]
        self.workers = int(workers)
        self.sims = []
        for m in self.members:
            cfg, fields = cases[m]
            if amg:
                cfg = dict(cfg, simulation=dict(cfg["simulation"], amg=dict(cfg["simulation"].get("amg", {}), **amg)))
            _, fl, _, sim = build_from_config(cfg, fields, device=self.device)
            sim._ensure_amg()
            sim._set_well_cells()
            fl.s_o = torch.empty_like(fl.s_w)
            self.sims.append(sim)
        self.last_stats: list[dict] = []
        self.last_span_ms = 0.0

    @property
    def local_cells(self) -> int:
        return sum(self.cells[m] for m in self.members)

    def run(self, steps: int, dt: float) -> list[dict]:
        """Advance every local member by `steps` steps of dt seconds."""
        n = len(self.sims)
        if n == 0:
            self.last_stats = []
            self.last_span_ms = 0.0
            return []
        for s in self.sims:
            s._sync_well_controls()
        P = C.c_void_p * n
        models = P(*[s._h.value for s in self.sims])
        amgs = P(*[s._amg_h.value for s in self.sims])
        arrs = {k: P(*[ptr(getattr(s.fluid, k)) for s in self.sims]) for k in ("pressure", "s_w", "s_g", "s_o")}
        cells = (C.c_int * n)(*[self.cells[m] for m in self.members])
        stats = (_lib.EnsembleMemberStats * n)()
        kp = self.sims[0].krylov_params()
        span = C.c_double(0.0)
        torch.cuda.synchronize(self.device)
        with torch.cuda.device(self.device):
            rc = lib.impes_ensemble_run(models, amgs, arrs["pressure"], arrs["s_w"], arrs["s_g"], arrs["s_o"],
                                        cells, n, int(steps), float(dt), C.byref(kp), self.workers, stats,
                                        C.byref(span))
        self.last_span_ms = span.value
        for s in self.sims:
            s._wells_stale = True
            s.step_count += steps
        self.last_stats = [{"member": m, "cells": self.cells[m], "status": st.status,
                            "steps": st.steps_done, "iterations": st.iterations,
                            "device_ms": st.device_ms, "worker": st.worker}
                           for m, st in zip(self.members, stats)]
        check(rc, "impes_ensemble_run")
        return self.last_stats

    def summary(self) -> list[dict]:
        """Per-member state summary (mean pressure in MPa, mean and max Sw) with the
        last run's statistics."""
        out = []
        for m, s, st in zip(self.members, self.sims, self.last_stats or [{}] * len(self.sims)):
            fl = s.fluid
            out.append(dict(st, member=m, p_mean_MPa=float(fl.pressure.mean()) / 1e6,
                            sw_mean=float(fl.s_w.mean()), sw_max=float(fl.s_w.max())))
        return out

    def close(self):
        for s in self.sims:
            s.close()
        self.sims = []
