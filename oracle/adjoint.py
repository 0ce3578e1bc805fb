"""Adjoint checker: a float64 torch restatement of the oracle's oil-water IMPES
step, differentiated by autograd.

TEST INFRASTRUCTURE ONLY.  Imported by tests/ and nothing on the product path.

The reference has no adjoint.  This module pins the hand-written CUDA adjoint
against autograd through a dense restatement of the reference's step:

* pressure step (simulation.py:867-904, 1546-1620): upwinded total mobility on
  the previous pressure, accumulation PV*ct/dt, rate and BHP wells
  (simulation.py:1622-1660), gravity on z faces; solved densely with
  ``torch.linalg.solve``;
* saturation step (simulation.py:968-1544) for oil-water without PVT and
  capillarity: upwinded water flux on the new pressure with the averaged-density
  gravity term, injector availability choke (simulation.py:1074-1115), BHP
  producer ``WI*lambda_t*(p - p_bhp)`` split by fractional flow, substep count
  from the saturation window, clamped equal increments;
* objective J = sum_t sum_producers (q_o - q_target)^2 with the producer oil
  rate in m3/day from the flux balance of the producer's pressure row
  q = sum_f c_f (p_nb - p_c) - PV*ct/dt*(p_c - p_prev) + Qg_c, times the oil
  fractional flow at the previous saturation.  (The well's own
  WI*lambda_t*(p_c - p_bhp) is the same number algebraically but is round-off:
  p_c sits within an ulp or so of p_bhp.)

Non-smooth points follow the taken branch: upwind directions, the substep count
and the availability choke's branch are fixed by the forward values; a clamp
passes the gradient when the unclamped value is inside or on its bounds.

The forward restates oracle/impes.py's ``Model.assemble``/``saturation`` for
this case; ``tests/test_adjoint_oracle.py`` checks the two agree.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .impes import G, Model

__all__ = ["TorchIMPES", "producer_rates", "objective"]


def _clampw(x, lo, hi):
    """min(max(x, lo), hi) with the gradient passed through on the bounds."""
    y = torch.where(x < lo, lo + 0.0 * x, x)
    return torch.where(y > hi, hi + 0.0 * y, y)


class TorchIMPES:
    """Dense float64 IMPES for an oil-water ``oracle.impes.Model`` configuration.

    ``lnk`` scales kx, ky and kz of each cell together (kx = exp(lnk) and the
    model's ky/kx and kz/kx ratios are kept); ``poro`` gives PV = V * poro.
    """

    def __init__(self, model: Model):
        m = model
        if m.pvt is not None or m.pc_scale != 0.0 or m.pc_og_scale != 0.0:
            raise ValueError("the adjoint covers oil-water without PVT or capillarity")
        if m.relperm_model != "corey":
            raise ValueError("the adjoint covers Corey relative permeability")
        if np.any(m.sg != 0.0):
            raise ValueError("the adjoint covers oil-water (s_g = 0)")
        self.m = m
        self.shape = (m.nx, m.ny, m.nz)
        kx = torch.tensor(m.kx, dtype=torch.float64)
        self.ry = torch.tensor(m.ky, dtype=torch.float64) / kx
        self.rz = torch.tensor(m.kz, dtype=torch.float64) / kx
        self.vol = (m.dx * m.dy) * m.dz
        self.lnk0 = torch.log(kx).reshape(-1)
        self.poro0 = torch.tensor(m.poro, dtype=torch.float64).reshape(-1)

    # -- fluid ------------------------------------------------------------
    def _mob(self, sw):
        m = self.m
        den = 1 - m.sw_cr - m.so_r
        s = _clampw((sw - m.sw_cr) / den, 0.0, 1.0)
        krw = s ** m.nw
        kro = (1 - s) ** m.no
        return krw / m.mu_water, kro / m.mu_oil

    def _rho(self, p):
        m = self.m
        return (m.rho_water_ref * (1.0 + m.c_w * (p - 1e5)),
                m.rho_oil_ref * (1.0 + m.c_o * (p - 1e5)))

    def _trans(self, lnk):
        m = self.m
        kx = torch.exp(lnk).reshape(self.shape)
        ky, kz = kx * self.ry, kx * self.rz

        def h(a, b):
            return 2 * a * b / (a + b + 1e-15)
        tx = h(kx[:-1], kx[1:]) * m.dy * m.dz / m.dx
        ty = h(ky[:, :-1], ky[:, 1:]) * m.dx * m.dz / m.dy
        tz = h(kz[:, :, :-1], kz[:, :, 1:]) * m.dx * m.dy / m.dz
        return tx, ty, tz

    @staticmethod
    def _up(dp, a, b):
        return torch.where(dp > 0, a, b)

    # -- one step ------------------------------------------------------------
    def step(self, p, sw, lnk, poro, dt):
        """(p_new, sw_new, producer oil rates [m3/d] of this step)."""
        m = self.m
        nx, ny, nz = self.shape
        N = nx * ny * nz
        tx, ty, tz = self._trans(lnk)
        pv = self.vol * poro
        mw, mo = self._mob(sw)
        mt = mw + mo
        P, Mt = p.reshape(self.shape), mt.reshape(self.shape)
        dpx = (P[:-1] - P[1:]).detach()
        dpy = (P[:, :-1] - P[:, 1:]).detach()
        dpz = (P[:, :, :-1] - P[:, :, 1:]).detach()
        cx = tx * self._up(dpx, Mt[:-1], Mt[1:])
        cy = ty * self._up(dpy, Mt[:, :-1], Mt[:, 1:])
        cz = tz * self._up(dpz, Mt[:, :, :-1], Mt[:, :, 1:])
        acc = pv * m.cf / dt
        idx = torch.arange(N).reshape(self.shape)
        A = torch.zeros(N, N, dtype=torch.float64)
        for a, b, c in ((idx[:-1], idx[1:], cx), (idx[:, :-1], idx[:, 1:], cy), (idx[:, :, :-1], idx[:, :, 1:], cz)):
            a, b, c = a.reshape(-1), b.reshape(-1), c.reshape(-1)
            A = A.index_put((a, b), -c, accumulate=True)
            A = A.index_put((b, a), -c, accumulate=True)
            A = A.index_put((a, a), c, accumulate=True)
            A = A.index_put((b, b), c, accumulate=True)
        diag = acc.clone()
        q = torch.zeros(N, dtype=torch.float64)
        rate_scale = float(m.sim_params.get("global_rate_scale", 1.0))
        prods = []
        for w in m.wells:
            c = m.cell(w)
            if w.control_type == "rate":
                if w.type == "producer" and w.bhp_min is not None:
                    raise ValueError("bhp_min producers are outside the adjoint")
                q = q.index_put((torch.tensor([c]),),
                                torch.tensor([(w.control_value * rate_scale) / 86400.0 * (1 if w.type == "injector" else -1)],
                                             dtype=torch.float64), accumulate=True)
            else:
                wd = w.well_index * mt[c]
                diag = diag.index_put((torch.tensor([c]),), wd.reshape(1), accumulate=True)
                q = q.index_put((torch.tensor([c]),), (wd * (w.control_value * 1e6)).reshape(1), accumulate=True)
            if w.type == "producer":
                prods.append(w)
        A = A + torch.diag(diag)
        Qg = torch.zeros(self.shape, dtype=torch.float64)
        if m.dz > 0 and nz > 1:
            Mw, Mo = mw.reshape(self.shape), mo.reshape(self.shape)
            rw, ro = (r.reshape(self.shape) for r in self._rho(p))
            up = dpz > 0
            gf = tz * G * m.dz * (torch.where(up, Mw[:, :, :-1], Mw[:, :, 1:]) * torch.where(up, rw[:, :, :-1], rw[:, :, 1:])
                                  + torch.where(up, Mo[:, :, :-1], Mo[:, :, 1:]) * torch.where(up, ro[:, :, :-1], ro[:, :, 1:]))
            Qg = torch.cat([torch.zeros(nx, ny, 1, dtype=torch.float64), gf], 2) \
                - torch.cat([gf, torch.zeros(nx, ny, 1, dtype=torch.float64)], 2)
        Qg = Qg.reshape(-1)
        b = acc * p + q + Qg
        p_new = torch.linalg.solve(A, b)

        # producer oil rates from the flux balance of each producer's row, built
        # from the face coefficients (A's row holds WI*lambda_t ~ 1e15 x c_f on the
        # diagonal; summing the row would cancel to round-off)
        fo = mo / (mt + 1e-10)
        Pn = p_new.reshape(self.shape)
        Fx = cx * (Pn[:-1] - Pn[1:])
        Fy = cy * (Pn[:, :-1] - Pn[:, 1:])
        Fz = cz * (Pn[:, :, :-1] - Pn[:, :, 1:])
        inflow = self._net_in(Fx, Fy, Fz)
        rates = []
        for w in prods:
            c = m.cell(w)
            qfb = inflow[c] - acc[c] * (p_new[c] - p[c]) + Qg[c]
            rates.append(qfb * fo[c] * 86400.0)

        sw_new = self._saturation(p_new, sw, tx, ty, tz, pv, dt)
        return p_new, sw_new, rates

    def _net_in(self, fx, fy, fz):
        """Per-cell sum of face flows f (positive from the lower to the higher index)
        into the cell: +f at the higher cell, -f at the lower one."""
        nx, ny, nz = self.shape
        z = torch.zeros
        d = (torch.cat([z(1, ny, nz, dtype=torch.float64), fx], 0) - torch.cat([fx, z(1, ny, nz, dtype=torch.float64)], 0)
             + torch.cat([z(nx, 1, nz, dtype=torch.float64), fy], 1) - torch.cat([fy, z(nx, 1, nz, dtype=torch.float64)], 1)
             + torch.cat([z(nx, ny, 1, dtype=torch.float64), fz], 2) - torch.cat([fz, z(nx, ny, 1, dtype=torch.float64)], 2))
        return d.reshape(-1)

    def _saturation(self, p, sw, tx, ty, tz, pv, dt):
        m = self.m
        nx, ny, nz = self.shape
        N = nx * ny * nz
        mw, mo = self._mob(sw)
        mt = mw + mo
        P, Mw = p.reshape(self.shape), mw.reshape(self.shape)
        dpx = P[:-1] - P[1:]
        dpy = P[:, :-1] - P[:, 1:]
        dpz = P[:, :, :-1] - P[:, :, 1:]
        ux, uy, uz = dpx.detach() > 0, dpy.detach() > 0, dpz.detach() > 0
        mwx = torch.where(ux, Mw[:-1], Mw[1:])
        mwy = torch.where(uy, Mw[:, :-1], Mw[:, 1:])
        mwz = torch.where(uz, Mw[:, :, :-1], Mw[:, :, 1:])
        if m.dz > 0 and nz > 1:
            rw = self._rho(p)[0].reshape(self.shape)
            pot_z = dpz + G * (0.5 * (rw[:, :, :-1] + rw[:, :, 1:])) * m.dz
        else:
            pot_z = dpz
        fx, fy, fz = tx * mwx * dpx, ty * mwy * dpy, tz * mwz * pot_z
        div = -self._net_in(fx, fy, fz)
        fw = mw / (mt + 1e-10)
        qw = torch.zeros(N, dtype=torch.float64)
        rate_scale = float(m.sim_params.get("global_rate_scale", 1.0))
        so_r, sw_min = float(m.so_r), float(m.sw_cr)
        for w in m.wells:
            if w.i >= m.nx or w.j >= m.ny or w.k >= m.nz:
                continue
            c = m.cell(w)
            if w.control_type == "rate":
                q_base = (w.control_value * rate_scale) / 86400.0
                q_total = q_base * (1 if w.type == "injector" else -1)
                if w.type == "injector":
                    if w.injected_phase == "gas":
                        raise ValueError("gas injection is outside the oil-water adjoint")
                    sw_up = torch.clamp((1.0 - so_r - 0.0) - sw[c], min=0.0)
                    dS = (dt / torch.clamp(pv[c], min=1e-12)) * q_total
                    if float(dS.detach()) > 0.0:
                        ratio = sw_up / torch.clamp(dS, min=1e-12)
                    else:
                        ratio = (sw[c] - sw_min) / torch.clamp(dS.abs(), min=1e-12)
                    alpha = ratio if float(ratio.detach()) < 1.0 else torch.ones((), dtype=torch.float64)
                    alpha = torch.clamp(alpha, 0.0, 1.0)
                    qw = qw.index_put((torch.tensor([c]),), (q_total * alpha).reshape(1), accumulate=True)
                else:
                    qw = qw.index_put((torch.tensor([c]),), (q_total * fw[c]).reshape(1), accumulate=True)
            else:
                q_total = w.well_index * mt[c] * (p[c] - w.control_value * 1e6)
                if w.type == "injector":
                    if w.injected_phase == "gas":
                        raise ValueError("gas injection is outside the oil-water adjoint")
                    qw = qw.index_put((torch.tensor([c]),), (-q_total).reshape(1), accumulate=True)
                else:
                    qw = qw.index_put((torch.tensor([c]),), (-q_total * fw[c]).reshape(1), accumulate=True)
        dSw = (dt / pv) * (qw - div)
        max_dS = m.sim_params.get("max_saturation_change", 0.05)
        eps = 1e-12
        d = dSw.detach().numpy()
        swo = sw.detach().numpy()
        sw_up = np.maximum(1.0 - so_r - swo, 0.0)
        sw_dn = np.maximum(swo - sw_min, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            rat_w = np.where(d > 0, d / np.maximum(sw_up, eps), (-d) / np.maximum(sw_dn, eps))
            rat = np.maximum(np.maximum(rat_w, 0.0), np.abs(d) / max_dS)
        rmax = rat.max()
        if not np.isfinite(rmax):
            rmax = 0.0
        n_sub = min(max(int(math.ceil(rmax)), 1), int(m.sim_params.get("max_substeps", 20)))
        inc = dSw / n_sub
        s = sw
        for _ in range(n_sub):
            s = _clampw(s + inc, float(m.sw_cr), 1.0 - so_r)
        return s


def producer_rates(model: Model, dt, steps, lnk=None, poro=None):
    """Producer oil rates [steps x producers] (m3/d) of a TorchIMPES forward run."""
    t = TorchIMPES(model)
    p = torch.tensor(model.p, dtype=torch.float64)
    sw = torch.tensor(model.sw, dtype=torch.float64)
    lnk = t.lnk0 if lnk is None else lnk
    poro = t.poro0 if poro is None else poro
    out = []
    for _ in range(steps):
        p, sw, r = t.step(p, sw, lnk, poro, dt)
        out.append(torch.stack(r))
    return torch.stack(out)


def objective(model: Model, dt, steps, target, lnk=None, poro=None):
    """J = sum (q_o - target)^2 and its gradients w.r.t. ln k and porosity (autograd)."""
    t = TorchIMPES(model)
    lnk = (t.lnk0 if lnk is None else torch.as_tensor(lnk, dtype=torch.float64)).clone().requires_grad_(True)
    poro = (t.poro0 if poro is None else torch.as_tensor(poro, dtype=torch.float64)).clone().requires_grad_(True)
    q = producer_rates(model, dt, steps, lnk, poro)
    J = ((q - torch.as_tensor(target, dtype=torch.float64)) ** 2).sum()
    g_lnk, g_poro = torch.autograd.grad(J, (lnk, poro))
    return float(J.detach()), g_lnk.numpy(), g_poro.numpy(), q.detach().numpy()
