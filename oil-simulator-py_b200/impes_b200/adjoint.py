"""History-matching adjoint on the B200 (no counterpart in the reference).

J(ln k, phi) = sum over steps and producers of (q_o - q_target)^2, with q_o the
producer oil rate in m3/day taken from the flux balance of the producer's
pressure row.  That is the reference's WI*lambda_t*(p - p_bhp)
(simulation.py:1297) without its round-off.  The forward run and the reverse
sweep are the library's CUDA kernels (``impes_adjoint_gradient``): checkpoints
every ``checkpoint_every`` steps, the adjoint pressure solve on the forward
hierarchy (A is symmetric), a reverse saturation sweep that replays the clamped
substeps.

``misfit(lnk, poro, ...)`` is a ``torch.autograd.Function``: its backward returns
the adjoint gradient.  Scope: oil-water without PVT or capillarity, Corey
relative permeability, no bhp_min switching.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .simulator import build_from_config

__all__ = ["producer_rates", "misfit_gradient", "misfit", "MisfitFunction"]


def _krylov(tol, restart=60, max_iters=2000, use_x0=1, precision="fp64"):
    prec = 1 if precision in ("mixed", "fp32") else 0
    return _lib.KrylovParams(float(tol), int(restart), int(max_iters), _lib.NORM_JACOBI, prec, int(use_x0))


def _with_precision(cfg, precision):
    """The configuration with its AMG hierarchy keeping fp32 levels when the
    solves use the fp32 V-cycle."""
    if precision == "fp64":
        return cfg
    sim = dict(cfg["simulation"])
    sim["amg"] = dict(sim.get("amg", {}), precision="mixed")
    return dict(cfg, simulation=sim)


def _fields(cfg, lnk, poro, ky_ratio, kz_ratio):
    kx = torch.exp(lnk.detach().to(torch.float64))
    return {"kx": kx, "ky": kx * ky_ratio, "kz": kx * kz_ratio, "poro": poro.detach().to(torch.float64)}


def _sim(cfg, fields, device):
    _, fl, _, sim = build_from_config(cfg, fields, device=device)
    sim._ensure_amg()
    return fl, sim


def _dt(cfg, dt):
    return float(dt) if dt is not None else float(cfg["simulation"]["time_step_days"]) * 86400.0


def producer_rates(cfg: dict, fields: dict, steps: int, dt: Optional[float] = None, *,
                   tol: float = 1e-11, device="cuda") -> np.ndarray:
    """Producer oil rates [steps, producers] (m3/day) of a forward run."""
    fl, sim = _sim(cfg, fields, device)
    try:
        n = C.c_int()
        check(lib.impes_adjoint_num_producers(sim._h, C.byref(n)), "impes_adjoint_num_producers")
        out = np.zeros((steps, n.value))
        p = fl.pressure.reshape(-1).contiguous().clone()
        sw = fl.s_w.reshape(-1).contiguous().clone()
        kp = _krylov(tol)
        check(lib.impes_adjoint_rates(sim._h, sim._amg_h, ptr(p), ptr(sw), int(steps), _dt(cfg, dt),
                                      C.byref(kp), out.ctypes.data if out.size else None,
                                      _lib.stream_of(sim.device)), "impes_adjoint_rates")
        return out
    finally:
        sim.close()


def misfit_gradient(cfg: dict, fields: dict, target, steps: int, dt: Optional[float] = None, *,
                    checkpoint_every: int = 10, tol: float = 1e-11, adjoint_tol: float = 1e-11,
                    device="cuda", precision: str = "fp64") -> dict:
    """J, dJ/dln k and dJ/dphi (device tensors shaped like the grid), the forward
    rates and the run statistics.  ``precision="mixed"`` runs the forward and
    adjoint FGMRES solves with the fp32 V-cycle (fp64 Krylov vectors)."""
    fl, sim = _sim(_with_precision(cfg, precision), fields, device)
    try:
        n = C.c_int()
        check(lib.impes_adjoint_num_producers(sim._h, C.byref(n)), "impes_adjoint_num_producers")
        target = np.ascontiguousarray(np.asarray(target, dtype=np.float64).reshape(steps, n.value))
        rates = np.zeros((steps, n.value))
        r = sim.reservoir
        g_lnk = torch.zeros(r.nx * r.ny * r.nz, dtype=torch.float64, device=sim.device)
        g_poro = torch.zeros_like(g_lnk)
        kx, ky, kz, _ = sim._rock
        p0 = fl.pressure.reshape(-1).contiguous()
        sw0 = fl.s_w.reshape(-1).contiguous()
        kf, ka = _krylov(tol, precision=precision), _krylov(adjoint_tol, use_x0=0, precision=precision)
        st = _lib.AdjointStats()
        check(lib.impes_adjoint_gradient(sim._h, sim._amg_h, ptr(p0), ptr(sw0), ptr(kx), ptr(ky), ptr(kz),
                                         int(steps), int(checkpoint_every), _dt(cfg, dt), C.byref(kf),
                                         C.byref(ka), target.ctypes.data, rates.ctypes.data, ptr(g_lnk),
                                         ptr(g_poro), C.byref(st), _lib.stream_of(sim.device)),
              "impes_adjoint_gradient")
        shape = (r.nx, r.ny, r.nz)
        stats = {k: getattr(st, k) for k, _ in _lib.AdjointStats._fields_}
        return {"J": st.J, "g_lnk": g_lnk.reshape(shape), "g_poro": g_poro.reshape(shape),
                "rates": rates, "stats": stats}
    finally:
        sim.close()


class MisfitFunction(torch.autograd.Function):
    """J(lnk, poro) with the adjoint gradient as its backward."""

    @staticmethod
    def forward(ctx, lnk, poro, cfg, target, steps, dt, ky_ratio, kz_ratio, opts):
        out = misfit_gradient(cfg, _fields(cfg, lnk, poro, ky_ratio, kz_ratio), target, steps, dt,
                              device=lnk.device, **opts)
        ctx.save_for_backward(out["g_lnk"].reshape(lnk.shape).to(lnk.dtype),
                              out["g_poro"].reshape(poro.shape).to(poro.dtype))
        return torch.tensor(out["J"], dtype=lnk.dtype, device=lnk.device)

    @staticmethod
    def backward(ctx, grad):
        g_lnk, g_poro = ctx.saved_tensors
        return grad * g_lnk, grad * g_poro, None, None, None, None, None, None, None


def misfit(lnk: torch.Tensor, poro: torch.Tensor, cfg: dict, target, steps: int,
           dt: Optional[float] = None, ky_ratio=1.0, kz_ratio=1.0, **opts) -> torch.Tensor:
    """Differentiable J for kx = exp(lnk), ky = kx*ky_ratio, kz = kx*kz_ratio (CUDA tensors
    shaped like the grid)."""
    return MisfitFunction.apply(lnk, poro, cfg, target, steps, dt, ky_ratio, kz_ratio, opts)
