"""IMPES simulator objects behind the reference's constructors and JSON schema.

Mirrors researchim-ai/oil-simulator-py:

* ``Reservoir`` (src/simulator/reservoir.py:4-80)
* ``Fluid``     (src/simulator/fluid.py:5-510) -- parameters, state tensors and the
  property functions the reference's tests call (``calc_oil_kr`` ...)
* ``PVTTable``  (src/simulator/pvt.py:5-64)
* ``Well`` / ``WellManager`` (src/simulator/well.py:5-132)
* ``Simulator`` (src/simulator/simulation.py:10-135, 822-1697) -- the IMPES step.

State tensors are float64 on the CUDA device, shaped (nx, ny, nz) with the flat
order c = (i*ny + j)*nz + k.  ``Simulator.run_step`` runs the whole IMPES step in
``libimpes_b200.so`` (assembly, AMG setup/update, pressure solve, saturation).
Heterogeneous rock is set, as with the reference, by assigning
``permeability_{x,y,z}`` / ``porosity`` / ``porous_volume`` on the Reservoir
before the Simulator is built.

Pressure solvers (``simulation.pressure_solver``): ``"amg"`` runs the reference's
stand-alone V-cycles with its stopping rule; ``"gmres_amg"`` runs FGMRES with one
V-cycle per iteration, ``simulation.amg.norm`` selecting
``"jacobi"`` (default) or ``"equilibrated"``, ``simulation.amg.precision``
``"fp64"`` or ``"mixed"`` (fp32 V-cycle), ``simulation.amg.max_iters`` the cap,
``simulation.amg.warm_start`` the first iterate: ``"extrapolate"`` (default, linear
in time from the last two steps), ``"quadratic"`` (from the last three),
``"previous"`` or ``false`` (zero).
Any other value, and a configuration without the key, runs the reference's
Jacobi-PCG (``cg_tolerance``, ``cg_max_iter``, absolute stopping test, one
relaxed retry), as the reference's own default does (simulation.py:905).  With a
BHP well that CG's absolute test on sqrt(r . D^-1 r) is dominated by the well row
and is not met, as in the reference; ``"gmres_amg"`` is the solver to choose.
AMG options beyond the reference's: ``simulation.amg.p_max_elements`` /
``p_trunc_factor`` (interpolation truncation), ``smoother`` (``"l1jacobi"`` or
``"chebyshev"``) and ``light_sweep_rows`` (levels of at most that many rows
smooth once before and once after their coarse correction).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .amg import ClassicalAMG, _cuda_device

MD_TO_M2 = 9.869233e-16
_PVT_COLS = ("pressure_MPa", "Bo", "Bw", "Bg", "mu_o_cP", "mu_w_cP", "mu_g_cP", "Rs_m3m3", "Rv_m3m3")


# ------------------------------------------------------------------- PVT
_LAYOUTS = {0: "csr", 1: "sell", 2: "dia", 3: "dia-tile"}

class PVTTable:
    """Black-oil table (``PVTTable``, pvt.py:18-64): columns linear in pressure (MPa)."""

    def __init__(self, json_path: Optional[str] = None, *, table: Optional[dict] = None):
        if table is None:
            with open(json_path, "r", encoding="utf-8") as f:
                table = json.load(f)
        self.P = np.asarray(table["pressure_MPa"], dtype=np.float64)
        self.Bo = np.asarray(table.get("Bo", []), dtype=np.float64)
        self.Bw = np.asarray(table.get("Bw", []), dtype=np.float64)
        self.Bg = np.asarray(table.get("Bg", []), dtype=np.float64)
        self.mu_o = np.asarray(table.get("mu_o_cP", []), dtype=np.float64)
        self.mu_w = np.asarray(table.get("mu_w_cP", []), dtype=np.float64)
        self.mu_g = np.asarray(table.get("mu_g_cP", []), dtype=np.float64)
        self.Rs = np.asarray(table.get("Rs_m3m3", []), dtype=np.float64)
        rv = table.get("Rv_m3m3")
        self.Rv = np.zeros_like(self.Rs) if rv is None else np.asarray(rv, dtype=np.float64)
        n = len(self.P)
        for arr, name in ((self.Bo, "Bo"), (self.Bw, "Bw"), (self.Bg, "Bg"), (self.mu_o, "mu_o_cP"),
                          (self.mu_w, "mu_w_cP"), (self.mu_g, "mu_g_cP"), (self.Rs, "Rs_m3m3"),
                          (self.Rv, "Rv_m3m3")):
            if len(arr) != n:
                raise ValueError(f"PVT: column length mismatch (pressure vs {name})")

    def packed(self) -> np.ndarray:
        """rows x 9 float64: P, Bo, Bw, Bg, mu_o, mu_w, mu_g, Rs, Rv (the C ABI layout)."""
        return np.ascontiguousarray(np.stack([self.P, self.Bo, self.Bw, self.Bg, self.mu_o, self.mu_w,
                                              self.mu_g, self.Rs, self.Rv], axis=1))

    def eval(self, P_MPa: np.ndarray) -> dict:
        p = np.asarray(P_MPa, dtype=np.float64)
        f = lambda fp: np.interp(p, self.P, fp, left=fp[0], right=fp[-1])  # noqa: E731
        return {"Bo": f(self.Bo), "Bw": f(self.Bw), "Bg": f(self.Bg), "mu_o": f(self.mu_o),
                "mu_w": f(self.mu_w), "mu_g": f(self.mu_g), "Rs": f(self.Rs), "Rv": f(self.Rv)}


# ------------------------------------------------------------- Reservoir
class Reservoir:
    """Grid and rock (``Reservoir``, reservoir.py:8-50)."""

    def __init__(self, config: dict, device=None):
        self.device = _cuda_device(device)
        self.dimensions = list(config.get("dimensions", [10, 10, 1]))
        self.nx, self.ny, self.nz = (int(v) for v in self.dimensions)
        gs = tuple(float(v) for v in config.get("grid_size", [10.0, 10.0, 10.0]))
        self.dx, self.dy, self.dz = gs
        porosity = config.get("porosity", 0.2)
        dims = (self.nx, self.ny, self.nz)
        kw = dict(device=self.device, dtype=torch.float64)
        self.porosity = torch.full(dims, float(porosity), **kw)
        k_h = config.get("permeability", 100.0)
        k_v = k_h * config.get("k_vertical_fraction", 0.1)
        self.permeability_x = torch.full(dims, k_h * MD_TO_M2, **kw)
        self.permeability_y = torch.full(dims, k_h * MD_TO_M2, **kw)
        self.permeability_z = torch.full(dims, k_v * MD_TO_M2, **kw)
        self.rock_compressibility = config.get("c_rock", 1e-5) / 1e6
        self.grid_size = torch.tensor(gs, **kw)
        self.cell_volume = (gs[0] * gs[1]) * gs[2]
        self.porous_volume = self.cell_volume * self.porosity

    @property
    def permeability_tensors(self):
        return self.permeability_x, self.permeability_y, self.permeability_z

    def get_cell_indices(self, i, j, k):
        """reservoir.py:70-80 (x-fastest; the IMPES path uses (i*ny + j)*nz + k)."""
        return i + j * self.nx + k * self.nx * self.ny


# ----------------------------------------------------------------- wells
class Well:
    """One well (``Well``, well.py:10-55).  ``last_*`` diagnostics are read from
    the device on access after a step."""

    def __init__(self, name, well_type, i, j, k, radius, control_type, control_value,
                 reservoir_dimensions, injected_phase="water", rate_type="reservoir",
                 surface_phase=None, limits=None, bhp_min=None):
        self.name, self.type = name, well_type
        self.i, self.j, self.k = int(i), int(j), int(k)
        self.radius = radius
        self.control_type, self.control_value = control_type, control_value
        self.injected_phase, self.rate_type, self.surface_phase = injected_phase, rate_type, surface_phase
        self.limits = limits or {}
        self.bhp_min = bhp_min
        nx, ny, nz = reservoir_dimensions
        self.cell_index = (self.i, self.j, self.k)
        self.cell_index_flat = self.i + self.j * nx + self.k * nx * ny   # well.py:40 (replaced per step)
        dx = dy = 1.0
        ro = 0.28 * ((dx ** 2 + dy ** 2) ** 0.5) / 2
        self.well_index = 2 * math.pi * 100.0 / (math.log(ro / radius) + 1e-12)
        self._sim = None
        self._idx = -1
        self._last = {"mode": None, "q": None, "rates": {}}

    def _refresh(self):
        if self._sim is not None:
            self._sim._refresh_wells()

    @property
    def last_q_total(self):
        self._refresh()
        return self._last["q"]

    @last_q_total.setter
    def last_q_total(self, v):
        self._last["q"] = v

    @property
    def last_surface_rates(self):
        self._refresh()
        return self._last["rates"]

    @last_surface_rates.setter
    def last_surface_rates(self, v):
        self._last["rates"] = v

    @property
    def last_mode(self):
        self._refresh()
        return self._last["mode"]

    @last_mode.setter
    def last_mode(self, v):
        self._last["mode"] = v

    def __str__(self):
        return (f"Well(name={self.name}, type={self.type}, pos=({self.i},{self.j},{self.k}), "
                f"control={self.control_type}:{self.control_value})")


class WellManager:
    """``WellManager`` (well.py:60-132): both coordinate/control schemas."""

    def __init__(self, well_configs, reservoir):
        self.wells = []
        for w in well_configs:
            if "coordinates" in w:
                i, j, k = w["coordinates"]
            elif "i" in w and "j" in w and "k" in w:
                i, j, k = w["i"], w["j"], w["k"]
            else:
                raise ValueError(f"invalid well coordinates: {w}")
            if "control" in w:
                ct, cv = w["control"]["type"], w["control"]["value"]
            elif "control_type" in w and "control_value" in w:
                ct, cv = w["control_type"], w["control_value"]
            else:
                raise ValueError(f"invalid well control: {w}")
            self.wells.append(Well(w["name"], w["type"], i, j, k, w["radius"], ct, cv, reservoir.dimensions,
                                   injected_phase=w.get("injected_phase", "water"),
                                   rate_type=w.get("rate_type", "reservoir"),
                                   surface_phase=w.get("surface_phase"), limits=w.get("limits"),
                                   bhp_min=w.get("bhp_min")))

    def get_wells(self):
        return self.wells

    def get_well_indices_flat(self):
        return torch.tensor([w.cell_index_flat for w in self.wells], dtype=torch.long)


# ----------------------------------------------------------------- fluid
class Fluid:
    """Fluid parameters and state (``Fluid``, fluid.py:10-126).  The property
    functions below are the reference's API for callers and tests; the IMPES
    step itself evaluates them inside the CUDA kernels."""

    def __init__(self, config: dict, reservoir: Reservoir, device=None):
        self.device = _cuda_device(device)
        self.dimensions = reservoir.dimensions
        dims = tuple(self.dimensions)
        kw = dict(device=self.device, dtype=torch.float64)
        initial_pressure = config.get("pressure", 20.0) * 1e6
        initial_sw = config.get("s_w", 0.2)
        initial_sg = config.get("s_g", 0.0)
        self.mu_oil = config.get("mu_oil", 1.0) * 1e-3
        self.mu_water = config.get("mu_water", 0.5) * 1e-3
        self.mu_gas = config.get("mu_gas", 0.02) * 1e-3
        self.rho_oil_ref = config.get("rho_oil", 850.0)
        self.rho_water_ref = config.get("rho_water", 1000.0)
        self.rho_gas_ref = config.get("rho_gas", 1.0)
        self.oil_compressibility = config.get("c_oil", 1e-5) / 1e6
        self.water_compressibility = config.get("c_water", 1e-5) / 1e6
        self.gas_compressibility = config.get("c_gas", 1e-3) / 1e6
        self.rock_compressibility = config.get("c_rock", 1e-5) / 1e6
        total_c = (self.oil_compressibility + self.water_compressibility + self.gas_compressibility
                   + self.rock_compressibility) / 3
        self.total_c = total_c
        self.cf = torch.full(dims, total_c, **kw)
        self.pvt = None
        pvt_cfg = config.get("pvt") if isinstance(config.get("pvt"), dict) else {}
        if "table" in pvt_cfg:
            self.pvt = PVTTable(table=pvt_cfg["table"])
        else:
            path = config.get("pvt_path") or pvt_cfg.get("path")
            if path:
                self.pvt = PVTTable(path)
        rp = config.get("relative_permeability", {})
        self.relperm_model = rp.get("model", "corey")
        self.nw, self.no, self.ng = rp.get("nw", 2), rp.get("no", 2), rp.get("ng", 2)
        self.ko_end_w, self.ko_end_g = rp.get("ko_end_w", 1.0), rp.get("ko_end_g", 1.0)
        self.now, self.nog = rp.get("now", float(self.no)), rp.get("nog", float(self.ng))
        self.krw_end, self.krg_end = rp.get("krw_end", 1.0), rp.get("krg_end", 1.0)
        self.sw_cr, self.so_r, self.sg_cr = rp.get("sw_cr", 0.2), rp.get("so_r", 0.2), rp.get("sg_cr", 0.0)
        self.pressure = torch.full(dims, float(initial_pressure), **kw)
        self.s_w = torch.full(dims, float(initial_sw), **kw)
        self.s_g = torch.full(dims, float(initial_sg), **kw)
        self.s_o = 1.0 - self.s_w - self.s_g
        if float((self.s_w + self.s_g).max()) > 1.0:
            raise ValueError("initial water + gas saturation exceeds 1")
        self.prev_pressure = self.pressure.clone()
        self.prev_sw = self.s_w.clone()
        self.prev_sg = self.s_g.clone()
        if "capillary_pressure" in config:
            pc = config["capillary_pressure"]
            self.pc_scale, self.pc_exponent = pc.get("pc_scale", 0.0), pc.get("pc_exponent", 1.5)
            self.pc_threshold = pc.get("pc_threshold", 0.01)
        else:
            self.pc_scale, self.pc_exponent = config.get("pc_scale", 0.0), config.get("pc_exponent", 1.5)
            self.pc_threshold = config.get("pc_threshold", 0.01)
        pcg = config.get("capillary_pressure_og", {})
        self.pc_og_scale, self.pc_og_exponent = pcg.get("pc_scale", 0.0), pcg.get("pc_exponent", 1.5)

    # reference property API (fluid.py:224-435); torch elementwise on the device
    def _get_normalized_saturation(self, s_w):
        return torch.clamp((s_w - self.sw_cr) / (1 - self.sw_cr - self.so_r), 0.0, 1.0)

    def calc_water_kr(self, s_w):
        return self._get_normalized_saturation(s_w) ** self.nw

    def calc_oil_kr(self, s_w, s_g=None):
        if self.relperm_model == "stone2":
            if s_g is None:
                s_g = self.s_g
            swn = torch.clamp((s_w - self.sw_cr) / (1.0 - self.sw_cr - self.so_r + 1e-12), 0.0, 1.0)
            sgn = torch.clamp((s_g - self.sg_cr) / (1.0 - self.sg_cr - self.so_r + 1e-12), 0.0, 1.0)
            kro = (self.ko_end_w * (1.0 - swn) ** self.now + self.ko_end_g * (1.0 - sgn) ** self.nog
                   - min(self.ko_end_w, self.ko_end_g))
            return torch.clamp(kro, min=0.0)
        return (1 - self._get_normalized_saturation(s_w)) ** self.no

    def calc_gas_kr(self, s_g):
        return torch.clamp(s_g / (1.0 - self.sw_cr - self.so_r + 1e-10), 0.0, 1.0) ** self.ng

    def get_rel_perms(self, s_w, s_g=None):
        kro = self.calc_oil_kr(s_w, s_g)
        krw = self.calc_water_kr(s_w)
        krg = self.calc_gas_kr(self.s_g if s_g is None else s_g)
        return kro, krw, krg

    def get_capillary_pressure(self, s_w):
        if self.pc_scale == 0.0:
            return torch.zeros_like(s_w)
        return self.pc_scale * (1.0 - self._get_normalized_saturation(s_w) + 1e-6) ** (-self.pc_exponent)

    def get_capillary_pressure_og(self, s_g):
        if self.pc_og_scale == 0.0:
            return torch.zeros_like(s_g)
        sgn = torch.clamp(s_g / (1 - self.sw_cr - self.so_r + 1e-12), 0.0, 1.0)
        return self.pc_og_scale * (1.0 - sgn + 1e-6) ** (-self.pc_og_exponent)

    calc_capillary_pressure = get_capillary_pressure

    def _eval_pvt(self, p_tensor: torch.Tensor, key: str) -> torch.Tensor:
        if self.pvt is None:
            raise RuntimeError("no PVT table loaded")
        vals = self.pvt.eval((p_tensor.detach().cpu().numpy() / 1e6).astype(np.float64))[key]
        return torch.from_numpy(vals).to(self.device, dtype=torch.float64).reshape(self.dimensions)

    def calc_water_density(self, pressure):
        if self.pvt is not None:
            return self.rho_water_ref / (self._eval_pvt(pressure, "Bw") + 1e-12)
        return self.rho_water_ref * (1.0 + self.water_compressibility * (pressure - 1e5))

    def calc_oil_density(self, pressure):
        if self.pvt is not None:
            return (self.rho_oil_ref + self._eval_pvt(pressure, "Rs") * self.rho_gas_ref) / (
                self._eval_pvt(pressure, "Bo") + 1e-12)
        return self.rho_oil_ref * (1.0 + self.oil_compressibility * (pressure - 1e5))

    def calc_gas_density(self, pressure):
        if self.pvt is not None:
            return (self.rho_gas_ref + self._eval_pvt(pressure, "Rv") * self.rho_oil_ref) / (
                self._eval_pvt(pressure, "Bg") + 1e-12)
        return self.rho_gas_ref * (1.0 + self.gas_compressibility * (pressure - 1e5))

    @property
    def rho_w(self):
        return self.calc_water_density(self.pressure)

    @property
    def rho_o(self):
        return self.calc_oil_density(self.pressure)

    @property
    def rho_g(self):
        return self.calc_gas_density(self.pressure)


# ------------------------------------------------------------- simulator
_SURF = {"oil": 0, "water": 1, "gas": 2, "liquid": 3}
_LIMS = (("wopr", 1), ("wlpr", 2), ("wgpr", 4), ("liqr", 8))


def model_desc(res: Reservoir, fl: Fluid, sim_params: dict) -> _lib.ModelDesc:
    d = _lib.ModelDesc()
    d.nx, d.ny, d.nz = res.nx, res.ny, res.nz
    d.dx, d.dy, d.dz = res.dx, res.dy, res.dz
    d.mu_o, d.mu_w, d.mu_g = fl.mu_oil, fl.mu_water, fl.mu_gas
    d.rho_o_ref, d.rho_w_ref, d.rho_g_ref = fl.rho_oil_ref, fl.rho_water_ref, fl.rho_gas_ref
    d.c_o, d.c_w = fl.oil_compressibility, fl.water_compressibility
    d.c_g, d.c_r = fl.gas_compressibility, fl.rock_compressibility
    d.cf = fl.total_c
    d.relperm_model = 1 if fl.relperm_model == "stone2" else 0
    d.nw, d.no, d.ng, d.now, d.nog = float(fl.nw), float(fl.no), float(fl.ng), float(fl.now), float(fl.nog)
    d.ko_end_w, d.ko_end_g = fl.ko_end_w, fl.ko_end_g
    d.sw_cr, d.so_r, d.sg_cr = fl.sw_cr, fl.so_r, fl.sg_cr
    d.pc_scale, d.pc_exponent = float(fl.pc_scale), float(fl.pc_exponent)
    d.pc_og_scale, d.pc_og_exponent = float(fl.pc_og_scale), float(fl.pc_og_exponent)
    d.gravity = 9.81
    d.global_rate_scale = float(sim_params.get("global_rate_scale", 1.0))
    d.max_saturation_change = float(sim_params.get("max_saturation_change", 0.05))
    d.max_substeps = int(sim_params.get("max_substeps", 20))
    d.pvt_rows = 0 if fl.pvt is None else len(fl.pvt.P)
    return d


def well_descs(wells) -> "C.Array":
    arr = (_lib.WellDesc * max(len(wells), 1))()
    for n, w in enumerate(wells):
        d = arr[n]
        d.i, d.j, d.k = w.i, w.j, w.k
        d.is_injector = 1 if w.type == "injector" else 0
        d.control_bhp = 1 if w.control_type == "bhp" else 0
        if w.control_type not in ("rate", "bhp"):
            raise ValueError(f"unknown control type {w.control_type!r}")
        d.value = float(w.control_value)
        d.well_index = float(w.well_index)
        d.injected_phase = 1 if w.injected_phase == "gas" else 0
        d.surface_rate = 1 if w.rate_type == "surface" else 0
        d.surface_phase = _SURF.get((w.surface_phase or "liquid").lower(), 3)
        mask = 0
        for q, (key, bit) in enumerate(_LIMS):
            if key in w.limits:
                mask |= bit
                d.limits[q] = float(w.limits[key])
        d.limit_mask = mask
        d.has_bhp_min = 0 if w.bhp_min is None else 1
        d.bhp_min = 0.0 if w.bhp_min is None else float(w.bhp_min)
    return arr


class Simulator:
    """IMPES simulator (``Simulator``, simulation.py:10-135) with the step on the B200."""

    def __init__(self, reservoir: Reservoir, fluid: Fluid, well_manager: WellManager, sim_params: dict,
                 device=None):
        self.reservoir, self.fluid, self.well_manager = reservoir, fluid, well_manager
        self.sim_params = sim_params
        self.device = _cuda_device(device)
        self.solver_type = sim_params.get("solver_type", "impes")
        if self.solver_type != "impes":
            raise NotImplementedError("only solver_type 'impes' is provided")
        self.g = 9.81
        self.porous_volume = reservoir.porous_volume
        amg_cfg = sim_params.get("amg", {}) or {}
        self.pressure_solver = sim_params.get("pressure_solver", "cg")   # simulation.py:905
        self.amg_tol = float(amg_cfg.get("tol", sim_params.get("cg_tolerance", 1e-6)))
        self.amg_max_cycles = int(amg_cfg.get("max_cycles", 20))
        self.amg_max_iters = int(amg_cfg.get("max_iters", 400))
        self.amg_restart = int(amg_cfg.get("restart", 60))
        # the reference's own stopping norm for its stand-alone V-cycles
        self.amg_norm = amg_cfg.get("norm", "equilibrated" if self.pressure_solver == "amg" else "jacobi")
        self.amg_precision = amg_cfg.get("precision", "fp64")
        # FGMRES's first iterate: the pressure extrapolated in time from the last
        # two steps ("extrapolate") or three ("quadratic"), the previous one
        # (True / "previous") or zero (False); the test stays ||r|| / ||b||
        ws = amg_cfg.get("warm_start", "extrapolate")
        self.amg_warm_start = ws if ws in ("extrapolate", "quadratic", "previous") else bool(ws)
        kw = dict(device=self.device, dtype=torch.float64)
        kx, ky, kz = (t.to(**kw).contiguous() for t in reservoir.permeability_tensors)
        poro = reservoir.porosity.to(**kw).contiguous()
        self._rock = (kx, ky, kz, poro)
        desc = model_desc(reservoir, fluid, sim_params)
        wells = well_manager.get_wells()
        self._wdesc = well_descs(wells)
        pvt = fluid.pvt.packed() if fluid.pvt is not None else None
        self._pvt_host = pvt
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.impes_model_create(C.byref(h), C.byref(desc), self._wdesc, len(wells),
                                         pvt.ctypes.data if pvt is not None else None,
                                         ptr(kx), ptr(ky), ptr(kz), ptr(poro),
                                         _lib.stream_of(self.device)), "impes_model_create")
        self._h = h
        self._well_values = [float(w.control_value) for w in wells]
        # porous volume as the library forms it (cell volume * porosity)
        self.porous_volume = reservoir.cell_volume * poro
        for n, w in enumerate(wells):
            w._sim, w._idx = self, n
        self._wells_stale = False
        self.amg: Optional[ClassicalAMG] = None
        self._amg_h = None
        self.last_krylov = {}
        self.last_substeps = 0
        self.step_count = 0

    def close(self):
        if getattr(self, "_h", None):
            lib.impes_model_destroy(self._h)
            self._h = None
        if getattr(self, "_amg_h", None):
            lib.impes_amg_destroy(self._amg_h)
            self._amg_h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------- stepping
    def _ensure_amg(self):
        if self._amg_h is None:
            amg_cfg = self.sim_params.get("amg", {}) or {}
            prm = _lib.AmgParams(float(amg_cfg.get("theta", 0.25)), int(amg_cfg.get("max_levels", 10)),
                                 int(amg_cfg.get("coarsest_size", 200)), 3, 0.6, 1e-6, 1e-6,
                                 int(amg_cfg.get("seed", 0)) & 0xFFFFFFFF,
                                 1 if self.amg_precision != "fp64" else 0,
                                 int(amg_cfg.get("p_max_elements", 0)),
                                 float(amg_cfg.get("p_trunc_factor", 0.0)),
                                 {"l1jacobi": 0, "chebyshev": 1}[amg_cfg.get("smoother", "l1jacobi")],
                                 float(amg_cfg.get("cheb_lower", 0.3)),
                                 int(amg_cfg.get("light_sweep_rows", 0)))
            h = C.c_void_p()
            check(lib.impes_amg_create(C.byref(h), C.byref(prm)), "impes_amg_create")
            self._amg_h = h

    def krylov_params(self) -> _lib.KrylovParams:
        norm = {"jacobi": _lib.NORM_JACOBI, "equilibrated": _lib.NORM_EQUILIBRATED}[self.amg_norm]
        prec = 1 if self.amg_precision in ("mixed", "fp32") else 0
        x0 = {False: 0, True: 1, "previous": 1, "extrapolate": 2, "quadratic": 3}[self.amg_warm_start]
        return _lib.KrylovParams(self.amg_tol, self.amg_restart, self.amg_max_iters, norm, prec, x0)

    def run_step(self, dt):
        """One time step (simulation.py:126-135)."""
        return self._impes_step(dt)

    def _set_well_cells(self):
        # simulation.py:1629-1630 replaces the x-fastest index with (i*ny + j)*nz + k
        r = self.reservoir
        for w in self.well_manager.get_wells():
            w.cell_index_flat = (w.i * r.ny + w.j) * r.nz + w.k

    def _sync_well_controls(self):
        """Upload Well.control_value when a caller changed it between steps (the
        reference reads it afresh every step, e.g. after rl_env.py:127-140)."""
        wells = self.well_manager.get_wells()
        vals = [float(w.control_value) for w in wells]
        if vals != self._well_values:
            arr = (C.c_double * max(len(vals), 1))(*vals)
            check(lib.impes_model_set_well_values(self._h, arr, len(vals), _lib.stream_of(self.device)),
                  "impes_model_set_well_values")
            self._well_values = vals

    def _impes_step(self, dt):
        """``_impes_step`` (simulation.py:822-865).  A pressure solve that misses its
        tolerance leaves the state untouched and is retried with dt divided by
        ``dt_reduction_factor``, up to ``max_time_step_attempts`` attempts."""
        self._ensure_amg()
        fl = self.fluid
        for name in ("pressure", "s_w", "s_g"):
            t = getattr(fl, name)
            if t.dtype != torch.float64 or t.device != self.device or not t.is_contiguous():
                setattr(fl, name, t.to(device=self.device, dtype=torch.float64).contiguous())
        if fl.s_o.dtype != torch.float64 or fl.s_o.device != self.device or not fl.s_o.is_contiguous():
            fl.s_o = torch.empty_like(fl.s_w)
        ks = _lib.KrylovStats()
        # "amg": the reference's stand-alone V-cycles; "gmres_amg": FGMRES with the
        # AMG V-cycle; any other value: the reference's Jacobi-PCG, as in
        # _impes_pressure_step (simulation.py:905-966)
        if self.pressure_solver == "amg":
            solver, kp = 0, self.krylov_params()
        elif self.pressure_solver == "gmres_amg":
            solver, kp = 1, self.krylov_params()
        else:
            solver = 2
            kp = _lib.KrylovParams(float(self.sim_params.get("cg_tolerance", 1e-6)), 0,
                                   int(self.sim_params.get("cg_max_iter", 500)), 0, 0, 0)
        max_attempts = int(self.sim_params.get("max_time_step_attempts", 5))
        factor = float(self.sim_params.get("dt_reduction_factor", 2.0))
        current_dt = float(dt)
        self._set_well_cells()
        self._sync_well_controls()
        for _ in range(max(1, max_attempts)):
            with torch.cuda.device(self.device):
                st = lib.impes_step(self._h, self._amg_h if solver != 2 else None, ptr(fl.pressure),
                                    ptr(fl.s_w), ptr(fl.s_g),
                                    ptr(fl.s_o), current_dt, solver, C.byref(kp), self.amg_max_cycles,
                                    C.byref(ks), None, _lib.stream_of(self.device))
            self.last_krylov = {"iterations": ks.iterations, "restarts": ks.restarts,
                                "converged": bool(ks.converged), "rel_res": ks.rel_res,
                                "true_rel_res": ks.true_rel_res, "dt": current_dt}
            if st == _lib.ERR_NOT_CONVERGED:
                current_dt /= factor
                continue
            check(st, "impes_step")
            fl.prev_pressure = fl.pressure.clone()
            fl.prev_sw = fl.s_w.clone()
            self._wells_stale = True
            self.step_count += 1
            return True
        return False

    # ------------------------------------------------------- diagnostics
    def _balances(self):
        st = _lib.SatStats()
        check(lib.impes_model_balances(self._h, C.byref(st), _lib.stream_of(self.device)))
        return st

    @property
    def mass_balance(self):
        st = self._balances()
        mb = list(st.mass_balance)
        self.last_substeps = st.substeps
        return {"water": {"in": mb[0], "out": mb[1]}, "oil": {"in": mb[2], "out": mb[3]},
                "gas": {"in": mb[4], "out": mb[5]}}

    @property
    def component_balance(self):
        cb = list(self._balances().component)
        return {"oil": {"in": cb[0], "out": cb[1], "accum": cb[2]},
                "gas": {"in": cb[3], "out": cb[4], "accum": cb[5]}}

    @property
    def substeps(self) -> int:
        return self._balances().substeps

    def _refresh_wells(self):
        if not self._wells_stale:
            return
        wells = self.well_manager.get_wells()
        if not wells:
            return
        arr = (_lib.WellState * len(wells))()
        check(lib.impes_well_states(self._h, arr, _lib.stream_of(self.device)))
        for w, st in zip(wells, arr):
            w._last["mode"] = {0: "rate", 1: "bhp"}.get(st.last_mode, w._last["mode"])
            if st.has_q_total:
                w._last["q"] = st.last_q_total
            if st.has_surface_rates:
                r = list(st.surface_rates)
                w._last["rates"] = {"oil": r[0], "water": r[1], "gas": r[2], "liquid": r[3]}
        cells = (C.c_int * len(wells))()
        check(lib.impes_well_cells(self._h, cells))
        for w, c in zip(wells, cells):
            w.cell_index_flat = int(c)
        self._wells_stale = False

    def amg_profile_levels(self, precision: str = "mixed", reps: int = 20):
        """Per-level device times (us) of one sweep, residual, restriction and
        prolongation of the pressure hierarchy (instrumentation)."""
        if self._amg_h is None:
            return []
        nl = C.c_int(0)
        check(lib.impes_amg_num_levels(self._amg_h, C.byref(nl)))
        out = (C.c_double * (4 * nl.value))()
        prec = 1 if precision in ("mixed", "fp32") else 0
        with torch.cuda.device(self.device):
            check(lib.impes_amg_profile_levels(self._amg_h, prec, int(reps), out, _lib.stream_of(self.device)),
                  "impes_amg_profile_levels")
        return [tuple(out[4 * l:4 * l + 4]) for l in range(nl.value)]

    def step_graphs(self):
        """(whole steps held as CUDA graphs, capture refused) of the pressure
        hierarchy (instrumentation)."""
        if self._amg_h is None:
            return (0, False)
        ng, bad = C.c_int(0), C.c_int(0)
        check(lib.impes_amg_step_graphs(self._amg_h, C.byref(ng), C.byref(bad)))
        return (ng.value, bool(bad.value))

    def amg_levels(self):
        """[(n, nnz, p_cols, p_nnz, is_coarsest, columns, lanes, layout)] of the
        pressure hierarchy; columns is the index storage of the level's sweeps:
        "i32", "u16" or "u16rel" (16-bit offsets from the row); lanes the
        autotuned lanes per row of the kernels on A, R and P (fp64 then fp32; 0:
        the default rule); layout (fp64, fp32) the storage the sweeps and
        residuals read: "csr", "sell", "dia" or "dia-tile" (the DIA copy of a grid's
        7-point stencil, two sweeps per launch on grid tiles)."""
        if self._amg_h is None:
            return []
        nl = C.c_int(0)
        check(lib.impes_amg_num_levels(self._amg_h, C.byref(nl)))
        out = []
        for l in range(nl.value):
            d = _lib.LevelDesc()
            check(lib.impes_amg_level_info(self._amg_h, l, C.byref(d)))
            cols = "i32" if d.col_index_bytes == 4 else ("u16rel" if d.col_row_relative else "u16")
            out.append((d.n, d.nnz, d.p_cols, d.p_nnz, bool(d.is_coarsest), cols, tuple(d.lanes),
                        tuple(_LAYOUTS[v] for v in d.layout)))
        return out

    # --------------------------------------------------- building blocks
    def csr_pattern(self):
        n, nnz = C.c_int(), C.c_int()
        check(lib.impes_model_nnz(self._h, C.byref(n), C.byref(nnz)))
        rowptr = torch.empty(n.value + 1, dtype=torch.int32, device=self.device)
        col = torch.empty(nnz.value, dtype=torch.int32, device=self.device)
        check(lib.impes_csr_pattern(self._h, ptr(rowptr), ptr(col), _lib.stream_of(self.device)))
        return rowptr, col

    def assemble(self, dt, p=None, s_w=None, s_g=None):
        """Pressure system (values in the static pattern, right-hand side) for the
        current (or given) state -- ``_impes_pressure_step`` steps 1-4."""
        fl = self.fluid
        p = (fl.pressure if p is None else p).to(self.device, torch.float64).contiguous()
        s_w = (fl.s_w if s_w is None else s_w).to(self.device, torch.float64).contiguous()
        s_g = (fl.s_g if s_g is None else s_g).to(self.device, torch.float64).contiguous()
        rowptr, col = self.csr_pattern()
        val = torch.empty(col.numel(), dtype=torch.float64, device=self.device)
        rhs = torch.empty(p.numel(), dtype=torch.float64, device=self.device)
        check(lib.impes_assemble(self._h, ptr(p), ptr(s_w), ptr(s_g), float(dt), ptr(val), ptr(rhs),
                                 _lib.stream_of(self.device)), "impes_assemble")
        self._set_well_cells()
        self._wells_stale = True
        return rowptr, col, val, rhs

    def saturation(self, p_new, dt):
        """Explicit saturation update in place on the fluid state (``_impes_saturation_step``)."""
        fl = self.fluid
        st = _lib.SatStats()
        p_new = p_new.to(self.device, torch.float64).contiguous()
        check(lib.impes_saturation(self._h, ptr(p_new), ptr(fl.s_w), ptr(fl.s_g), ptr(fl.s_o), float(dt),
                                   C.byref(st), _lib.stream_of(self.device)), "impes_saturation")
        self.last_substeps = st.substeps
        self._wells_stale = True
        return st.substeps

    def run(self, output_filename, save_vtk=False, results_root="results"):
        """Full run (simulation.py:2121-2260): total_time_days / time_step_days steps
        of run_step, intermediate states every save_interval steps, then the
        summary text and the npz of the final fields in
        results/<output_filename>_<timestamp>/.  Returns that directory."""
        from . import results as res
        total_days = self.sim_params.get("total_time_days", 100)
        step_days = self.sim_params.get("time_step_days", 1.0)
        save_interval = self.sim_params.get("save_interval", 10)
        num_steps = int(total_days / step_days)
        out_dir = res.results_dir(output_filename, results_root)
        inter = os.path.join(out_dir, "intermediate")
        if save_interval < num_steps:
            os.makedirs(inter, exist_ok=True)
        fl = self.fluid
        for i in range(num_steps):
            if not self.run_step(step_days * 86400):
                break
            if (i + 1) % save_interval == 0 and save_interval < num_steps:
                res.write_snapshot(os.path.join(inter, f"{output_filename}_step_{i+1}.npz"),
                                   fl.pressure.cpu().numpy(), fl.s_w.cpu().numpy(), fl.s_g.cpu().numpy())
        p, sw, sg = fl.pressure.cpu().numpy(), fl.s_w.cpu().numpy(), fl.s_g.cpu().numpy()
        so = fl.s_o.cpu().numpy().reshape(p.shape)
        res.write_summary(os.path.join(out_dir, f"{output_filename}.txt"), p, sw, sg, so, self.mass_balance,
                          bool(self.sim_params.get("write_full_arrays_txt", False)))
        if self.sim_params.get("save_npz", True):
            res.write_npz(os.path.join(out_dir, f"{output_filename}.npz"), p, sw, sg, so)
        if save_vtk:
            print("VTK output is not part of this package; the npz holds the final fields.")
        return out_dir

    def static_fields(self):
        """(Tx, Ty, Tz, PV) device tensors as the library computed them."""
        r = self.reservoir
        tx = torch.empty(max((r.nx - 1) * r.ny * r.nz, 0), dtype=torch.float64, device=self.device)
        ty = torch.empty(max(r.nx * (r.ny - 1) * r.nz, 0), dtype=torch.float64, device=self.device)
        tz = torch.empty(max(r.nx * r.ny * (r.nz - 1), 0), dtype=torch.float64, device=self.device)
        pv = torch.empty(r.nx * r.ny * r.nz, dtype=torch.float64, device=self.device)
        check(lib.impes_model_export_static(self._h, ptr(tx) if tx.numel() else None,
                                            ptr(ty) if ty.numel() else None,
                                            ptr(tz) if tz.numel() else None, ptr(pv),
                                            _lib.stream_of(self.device)))
        return tx, ty, tz, pv


def build_from_config(cfg: dict, fields: Optional[dict] = None, device=None):
    """(Reservoir, Fluid, WellManager, Simulator) from a config dict in the
    reference's schema, with optional heterogeneous rock ``fields``
    (kx, ky, kz in m^2, poro; arrays shaped (nx, ny, nz))."""
    res = Reservoir(cfg["reservoir"], device)
    if fields is not None:
        kw = dict(device=res.device, dtype=torch.float64)

        def field(v):
            t = v.detach().to(**kw) if torch.is_tensor(v) else torch.as_tensor(np.asarray(v), **kw)
            return t.reshape(res.nx, res.ny, res.nz)
        res.permeability_x = field(fields["kx"])
        res.permeability_y = field(fields["ky"])
        res.permeability_z = field(fields["kz"])
        res.porosity = field(fields["poro"])
        res.porous_volume = res.cell_volume * res.porosity
    wm = WellManager(cfg.get("wells", []), res)
    fl = Fluid(cfg["fluid"], res, device)
    sim = Simulator(res, fl, wm, cfg.get("simulation", {}), device)
    return res, fl, wm, sim
