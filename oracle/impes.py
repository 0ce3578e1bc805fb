"""Float64 CPU restatement of the reference's IMPES step (checker only).

Follows researchim-ai/oil-simulator-py:

* ``src/simulator/simulation.py`` -- transmissibilities (:52-74), the IMPES
  driver (:822-865), pressure step (:867-929), saturation step (:968-1544),
  matrix (:1546-1580), right-hand side (:1582-1620), well terms (:1622-1660);
* ``src/simulator/fluid.py`` -- relative permeability (:224-248, :377-435),
  densities (:129-158, :330-375), total compressibility (:190-222), capillary
  pressure (:273-296), PVT evaluation (:182-188);
* ``src/simulator/pvt.py:48-64`` -- ``np.interp`` with flat extrapolation;
* ``src/simulator/well.py:10-132`` -- Peaceman index and the two well schemas.

Layout: every field is a flat float64 array over cells ordered
``c = (i*ny + j)*nz + k`` (z fastest, ``simulation.py:804-816``).  The floating
point operation order of each expression follows the reference's so that the
restatement agrees with the reference run in float64 to the last bits wherever
the reference's arithmetic is elementwise.

The pressure linear solve is pluggable: ``solve='direct'`` (scipy spsolve, the
trajectory oracle) or any callable ``f(A_csr, b) -> x``.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

G = 9.81                    # simulation.py:81
MD_TO_M2 = 9.869233e-16     # reservoir.py:35


def tpow(x, e):
    """``tensor ** e`` with the special cases torch takes for a scalar exponent.

    torch evaluates ``x**2`` as ``x*x``, ``x**3`` as ``x*x*x``, ``x**-0.5`` as
    ``1/sqrt(x)``, ``x**-1`` as ``1/x`` and ``x**-2`` as ``1/(x*x)``; other
    exponents go through a general ``pow`` (which differs from libm's in the last
    bit, so those agree to round-off only).
    """
    e = float(e)
    if e == 0.0:
        return np.ones_like(x)
    if e == 1.0:
        return x.copy()
    if e == 2.0:
        return x * x
    if e == 3.0:
        return x * x * x
    if e == -0.5:
        return 1.0 / np.sqrt(x)
    if e == -1.0:
        return 1.0 / x
    if e == -2.0:
        return 1.0 / (x * x)
    return np.power(x, e)


# --------------------------------------------------------------------------- PVT
class PVT:
    """``PVTTable`` (pvt.py:18-64): columns interpolated by ``np.interp`` in MPa."""

    KEYS = ("Bo", "Bw", "Bg", "mu_o", "mu_w", "mu_g", "Rs", "Rv")

    def __init__(self, table: dict):
        self.P = np.asarray(table["pressure_MPa"], dtype=np.float64)
        cols = {
            "Bo": table.get("Bo", []), "Bw": table.get("Bw", []), "Bg": table.get("Bg", []),
            "mu_o": table.get("mu_o_cP", []), "mu_w": table.get("mu_w_cP", []),
            "mu_g": table.get("mu_g_cP", []), "Rs": table.get("Rs_m3m3", []),
        }
        self.cols = {k: np.asarray(v, dtype=np.float64) for k, v in cols.items()}
        rv = table.get("Rv_m3m3")
        self.cols["Rv"] = (np.zeros_like(self.cols["Rs"]) if rv is None
                           else np.asarray(rv, dtype=np.float64))
        for k, v in self.cols.items():
            if len(v) != len(self.P):
                raise ValueError(f"PVT: column {k} length mismatch")

    def eval(self, p_pa: np.ndarray, key: str) -> np.ndarray:
        # fluid.py:186-188 (float64 variant): p/1e6 then np.interp (pvt.py:48-50)
        fp = self.cols[key]
        return np.interp(p_pa / 1e6, self.P, fp, left=fp[0], right=fp[-1])


def load_pvt(fluid_cfg: dict, pvt_table: dict | None):
    """PVT from an explicit table, ``fluid.pvt.table``, or ``pvt_path``/``pvt.path`` (fluid.py:52-58)."""
    if pvt_table is not None:
        return PVT(pvt_table)
    if isinstance(fluid_cfg.get("pvt"), dict) and "table" in fluid_cfg["pvt"]:
        return PVT(fluid_cfg["pvt"]["table"])
    path = fluid_cfg.get("pvt_path") or fluid_cfg.get("pvt", {}).get("path")
    if path:
        with open(path, "r", encoding="utf-8") as f:
            return PVT(json.load(f))
    return None


# ------------------------------------------------------------------------- wells
@dataclass
class Well:
    name: str
    type: str
    i: int
    j: int
    k: int
    radius: float
    control_type: str
    control_value: float
    injected_phase: str = "water"
    rate_type: str = "reservoir"
    surface_phase: str | None = None
    limits: dict = field(default_factory=dict)
    bhp_min: float | None = None
    well_index: float = 0.0
    last_q_total: float | None = None
    last_surface_rates: dict = field(default_factory=dict)
    last_mode: str | None = None


def parse_wells(well_cfgs) -> list[Well]:
    """``WellManager.__init__`` (well.py:60-92) and ``Well.__init__`` (well.py:10-55)."""
    out = []
    for w in well_cfgs:
        if "coordinates" in w:
            i, j, k = w["coordinates"]
        elif "i" in w and "j" in w and "k" in w:
            i, j, k = w["i"], w["j"], w["k"]
        else:
            raise ValueError(f"bad well coordinates: {w}")
        if "control" in w:
            ct, cv = w["control"]["type"], w["control"]["value"]
        elif "control_type" in w and "control_value" in w:
            ct, cv = w["control_type"], w["control_value"]
        else:
            raise ValueError(f"bad well control: {w}")
        dx = dy = 1.0                                   # well.py:44
        ro = 0.28 * ((dx ** 2 + dy ** 2) ** 0.5) / 2    # well.py:47
        wi = 2 * math.pi * 100.0 / (math.log(ro / w["radius"]) + 1e-12)  # well.py:50-51
        out.append(Well(w["name"], w["type"], int(i), int(j), int(k), w["radius"], ct, cv,
                        w.get("injected_phase", "water"), w.get("rate_type", "reservoir"),
                        w.get("surface_phase"), w.get("limits") or {}, w.get("bhp_min"), wi))
    return out


# ------------------------------------------------------------------------- model
class Model:
    """The reference's ``Reservoir`` + ``Fluid`` + ``WellManager`` + IMPES ``Simulator``.

    ``kx, ky, kz`` (m^2) and ``poro`` optionally override the homogeneous fields
    the JSON schema can express (the harness does the same to the reference by
    assigning the tensors after ``Reservoir()`` and before ``Simulator()``).
    """

    def __init__(self, cfg: dict, kx=None, ky=None, kz=None, poro=None, pvt_table=None):
        rc, fc, sc = cfg["reservoir"], cfg["fluid"], cfg.get("simulation", {})
        self.sim_params = sc
        self.nx, self.ny, self.nz = [int(v) for v in rc.get("dimensions", [10, 10, 1])]
        nx, ny, nz = self.nx, self.ny, self.nz
        self.N = nx * ny * nz
        self.dx, self.dy, self.dz = [float(v) for v in rc.get("grid_size", [10.0, 10.0, 10.0])]
        shape = (nx, ny, nz)
        # reservoir.py:26-50
        porosity = rc.get("porosity", 0.2)
        k_h = rc.get("permeability", 100.0)
        k_v = k_h * rc.get("k_vertical_fraction", 0.1)
        self.kx = np.full(shape, k_h * MD_TO_M2) if kx is None else np.asarray(kx, np.float64).reshape(shape)
        self.ky = np.full(shape, k_h * MD_TO_M2) if ky is None else np.asarray(ky, np.float64).reshape(shape)
        self.kz = np.full(shape, k_v * MD_TO_M2) if kz is None else np.asarray(kz, np.float64).reshape(shape)
        self.poro = np.full(shape, porosity, dtype=np.float64) if poro is None else np.asarray(poro, np.float64).reshape(shape)
        cell_volume = (self.dx * self.dy) * self.dz     # reservoir.py:48-49 (tensor prod)
        self.pv = (cell_volume * self.poro).reshape(-1)  # reservoir.py:50

        # fluid.py:26-110
        self.p0 = fc.get("pressure", 20.0) * 1e6
        self.mu_oil = fc.get("mu_oil", 1.0) * 1e-3
        self.mu_water = fc.get("mu_water", 0.5) * 1e-3
        self.mu_gas = fc.get("mu_gas", 0.02) * 1e-3
        self.rho_oil_ref = fc.get("rho_oil", 850.0)
        self.rho_water_ref = fc.get("rho_water", 1000.0)
        self.rho_gas_ref = fc.get("rho_gas", 1.0)
        self.c_o = fc.get("c_oil", 1e-5) / 1e6
        self.c_w = fc.get("c_water", 1e-5) / 1e6
        self.c_g = fc.get("c_gas", 1e-3) / 1e6
        self.c_r = fc.get("c_rock", 1e-5) / 1e6
        self.cf = (self.c_o + self.c_w + self.c_g + self.c_r) / 3   # fluid.py:47
        self.pvt = load_pvt(fc, pvt_table)
        rp = fc.get("relative_permeability", {})
        self.relperm_model = rp.get("model", "corey")
        self.nw, self.no, self.ng = rp.get("nw", 2), rp.get("no", 2), rp.get("ng", 2)
        self.ko_end_w, self.ko_end_g = rp.get("ko_end_w", 1.0), rp.get("ko_end_g", 1.0)
        self.now, self.nog = rp.get("now", float(self.no)), rp.get("nog", float(self.ng))
        self.sw_cr, self.so_r, self.sg_cr = rp.get("sw_cr", 0.2), rp.get("so_r", 0.2), rp.get("sg_cr", 0.0)
        if "capillary_pressure" in fc:
            pc = fc["capillary_pressure"]
            self.pc_scale, self.pc_exponent = pc.get("pc_scale", 0.0), pc.get("pc_exponent", 1.5)
        else:
            self.pc_scale, self.pc_exponent = fc.get("pc_scale", 0.0), fc.get("pc_exponent", 1.5)
        pcg = fc.get("capillary_pressure_og", {})
        self.pc_og_scale, self.pc_og_exponent = pcg.get("pc_scale", 0.0), pcg.get("pc_exponent", 1.5)

        self.wells = parse_wells(cfg.get("wells", []))
        # simulation.py:52-74
        kxa, kya, kza = self.kx, self.ky, self.kz
        self.Tx = (2 * kxa[:-1] * kxa[1:] / (kxa[:-1] + kxa[1:] + 1e-15)) * self.dy * self.dz / self.dx
        self.Ty = (2 * kya[:, :-1] * kya[:, 1:] / (kya[:, :-1] + kya[:, 1:] + 1e-15)) * self.dx * self.dz / self.dy
        self.Tz = (2 * kza[:, :, :-1] * kza[:, :, 1:] / (kza[:, :, :-1] + kza[:, :, 1:] + 1e-15)) * self.dx * self.dy / self.dz
        # state (fluid.py:78-89)
        self.p = np.full(self.N, self.p0)
        self.sw = np.full(self.N, float(fc.get("s_w", 0.2)))
        self.sg = np.full(self.N, float(fc.get("s_g", 0.0)))
        self.so = (1.0 - self.sw) - self.sg
        self.mass_balance = {ph: {"in": 0.0, "out": 0.0} for ph in ("water", "oil", "gas")}
        self.component_balance = {"oil": {"in": 0.0, "out": 0.0, "accum": 0.0},
                                  "gas": {"in": 0.0, "out": 0.0, "accum": 0.0}}
        self.last_substeps = 0

    # ----------------------------------------------------------- fluid helpers
    def shape(self, v):
        return v.reshape(self.nx, self.ny, self.nz)

    def ev(self, p, key):
        return self.pvt.eval(p, key)

    def relperms(self, sw, sg):
        """(kro, krw, krg) -- ``Fluid.get_rel_perms`` (fluid.py:231-248, 377-435)."""
        s_norm = np.clip((sw - self.sw_cr) / (1 - self.sw_cr - self.so_r), 0.0, 1.0)
        krw = tpow(s_norm, self.nw)
        if self.relperm_model == "stone2":
            denom_w = 1.0 - self.sw_cr - self.so_r
            swn = np.clip((sw - self.sw_cr) / (denom_w + 1e-12), 0.0, 1.0)
            denom_g = 1.0 - self.sg_cr - self.so_r
            sgn = np.clip((sg - self.sg_cr) / (denom_g + 1e-12), 0.0, 1.0)
            krow = self.ko_end_w * tpow(1.0 - swn, self.now)
            krog = self.ko_end_g * tpow(1.0 - sgn, self.nog)
            kro = np.maximum(krow + krog - min(self.ko_end_w, self.ko_end_g), 0.0)
        else:
            kro = tpow(1 - s_norm, self.no)
        sgn2 = np.clip(sg / (1.0 - self.sw_cr - self.so_r + 1e-10), 0.0, 1.0)
        krg = tpow(sgn2, self.ng)
        return kro, krw, krg

    def viscosities(self, p):
        """(mu_o, mu_w, mu_g) in Pa*s -- ``simulation.py:875-877, 974-976``."""
        if self.pvt is not None:
            return self.ev(p, "mu_o") * 1e-3, self.ev(p, "mu_w") * 1e-3, self.ev(p, "mu_g") * 1e-3
        return self.mu_oil, self.mu_water, self.mu_gas

    def densities(self, p):
        """(rho_w, rho_o, rho_g) -- ``fluid.py:129-158, 330-375``."""
        if self.pvt is None:
            return (self.rho_water_ref * (1.0 + self.c_w * (p - 1e5)),
                    self.rho_oil_ref * (1.0 + self.c_o * (p - 1e5)),
                    self.rho_gas_ref * (1.0 + self.c_g * (p - 1e5)))
        bw, bo, rs, bg, rv = (self.ev(p, k) for k in ("Bw", "Bo", "Rs", "Bg", "Rv"))
        return (self.rho_water_ref / (bw + 1e-12),
                (self.rho_oil_ref + rs * self.rho_gas_ref) / (bo + 1e-12),
                (self.rho_gas_ref + rv * self.rho_oil_ref) / (bg + 1e-12))

    def total_compressibility(self, p, sw, sg):
        """``calc_total_compressibility`` (fluid.py:190-222)."""
        if self.pvt is None:
            return np.full(self.N, self.cf)
        P_mpa = p / 1e6
        Pp, Pm = P_mpa + 0.1, P_mpa - 0.1
        x0, xp, xm = P_mpa * 1e6, Pp * 1e6, Pm * 1e6
        B = {k: self.ev(x0, k) for k in ("Bw", "Bo", "Bg")}
        Bp = {k: self.ev(xp, k) for k in ("Bw", "Bo", "Bg")}
        Bm = {k: self.ev(xm, k) for k in ("Bw", "Bo", "Bg")}
        c = {k: -(((Bp[k] - Bm[k]) / (2 * 0.1)) / (B[k] + 1e-12)) / 1e6 for k in B}
        s_o = 1.0 - sw - sg
        return self.c_r + sw * c["Bw"] + s_o * c["Bo"] + sg * c["Bg"]

    def capillary(self, sw):
        """``get_capillary_pressure`` (fluid.py:273-287)."""
        if self.pc_scale == 0.0:
            return np.zeros_like(sw)
        s_norm = np.clip((sw - self.sw_cr) / (1 - self.sw_cr - self.so_r), 0.0, 1.0)
        return self.pc_scale * tpow(1.0 - s_norm + 1e-6, -self.pc_exponent)

    def capillary_og(self, sg):
        """``get_capillary_pressure_og`` (fluid.py:288-296)."""
        if self.pc_og_scale == 0.0:
            return np.zeros_like(sg)
        denom = 1 - self.sw_cr - self.so_r
        sgn = np.clip(sg / (denom + 1e-12), 0.0, 1.0)
        return self.pc_og_scale * tpow(1.0 - sgn + 1e-6, -self.pc_og_exponent)

    def cell(self, w):
        return (w.i * self.ny + w.j) * self.nz + w.k   # simulation.py:816

    # ------------------------------------------------------------- CSR pattern
    def csr_pattern(self):
        """Sorted 7-point CSR pattern after ``coalesce().to_sparse_csr()``.

        ``_build_pressure_matrix_vectorized`` (simulation.py:1546-1580) emits
        (row, col) pairs for x/y/z faces in both directions plus the diagonal;
        coalesce sorts them row-major, so each row holds, in column order,
        x-, y-, z-, diagonal, z+, y+, x+ (those that exist).
        """
        nx, ny, nz = self.nx, self.ny, self.nz
        idx = np.arange(self.N).reshape(nx, ny, nz)
        rows, cols = [], []
        for a, b in ((idx[:-1], idx[1:]), (idx[:, :-1], idx[:, 1:]), (idx[:, :, :-1], idx[:, :, 1:])):
            rows += [a.ravel(), b.ravel()]
            cols += [b.ravel(), a.ravel()]
        rows.append(idx.ravel()); cols.append(idx.ravel())
        r = np.concatenate(rows); c = np.concatenate(cols)
        order = np.lexsort((c, r))
        r, c = r[order], c[order]
        rowptr = np.zeros(self.N + 1, dtype=np.int64)
        np.add.at(rowptr, r + 1, 1)
        return np.cumsum(rowptr), c.astype(np.int64)

    # ---------------------------------------------------------- pressure step
    def assemble(self, dt):
        """(A csr float64, b, info) for the current state -- simulation.py:867-904."""
        nx, ny, nz, N = self.nx, self.ny, self.nz, self.N
        P = self.shape(self.p)
        kro, krw, krg = self.relperms(self.sw, self.sg)
        mu_o, mu_w, mu_g = self.viscosities(self.p)
        mob_w = krw / mu_w
        mob_o = kro / mu_o
        mob_g = krg / mu_g
        mob_t = mob_w + mob_o + mob_g
        Mt = self.shape(mob_t)
        dpx = P[:-1] - P[1:]
        dpy = P[:, :-1] - P[:, 1:]
        dpz = P[:, :, :-1] - P[:, :, 1:]
        Txt = self.Tx * np.where(dpx > 0, Mt[:-1], Mt[1:])
        Tyt = self.Ty * np.where(dpy > 0, Mt[:, :-1], Mt[:, 1:])
        Tzt = self.Tz * np.where(dpz > 0, Mt[:, :, :-1], Mt[:, :, 1:])
        q_wells, well_diag = self.well_terms(mob_t)
        # _build_pressure_matrix_vectorized (simulation.py:1546-1580)
        idx = np.arange(N).reshape(nx, ny, nz)
        seg_r, seg_c, seg_v = [], [], []
        for a, b, t in ((idx[:-1], idx[1:], Txt), (idx[:, :-1], idx[:, 1:], Tyt), (idx[:, :, :-1], idx[:, :, 1:], Tzt)):
            seg_r += [a.ravel(), b.ravel()]
            seg_c += [b.ravel(), a.ravel()]
            seg_v += [-t.ravel(), -t.ravel()]
        rows = np.concatenate(seg_r); cols = np.concatenate(seg_c); vals = np.concatenate(seg_v)
        ct = self.total_compressibility(self.p, self.sw, self.sg)
        acc = self.pv * ct / dt
        diag = np.zeros(N)
        for r_, v_ in zip(seg_r, seg_v):          # scatter_add_ in segment order
            diag[r_] += -v_
        diag += acc
        diag += well_diag
        A = sp.csr_matrix((np.concatenate([vals, diag]),
                           (np.concatenate([rows, idx.ravel()]), np.concatenate([cols, idx.ravel()]))),
                          shape=(N, N))
        A.sort_indices()
        b = self.rhs(dt, mob_w, mob_o, mob_g, q_wells, dpx, dpy, dpz, ct)
        return A, b, {"mob_t": mob_t, "diag": diag}

    def well_terms(self, mob_t):
        """``_calculate_well_terms`` (simulation.py:1622-1660)."""
        q = np.zeros(self.N)
        wd = np.zeros(self.N)
        rate_scale = float(self.sim_params.get("global_rate_scale", 1.0))
        for w in self.wells:
            c = self.cell(w)
            if w.control_type == "rate":
                rate_si = (w.control_value * rate_scale) / 86400.0 * (1 if w.type == "injector" else -1)
                if w.type == "producer" and w.bhp_min is not None:
                    p_block, mt = self.p[c], mob_t[c]
                    denom = w.well_index * mt + 1e-12
                    p_req = p_block - rate_si / denom
                    p_min = w.bhp_min * 1e6
                    if p_req < p_min:
                        w.last_mode = "bhp"
                        wd[c] += w.well_index * mt
                        q[c] += w.well_index * mt * p_min
                        continue
                w.last_mode = "rate"
                q[c] += rate_si
            elif w.control_type == "bhp":
                mt = mob_t[c]
                wd[c] += w.well_index * mt
                q[c] += w.well_index * mt * (w.control_value * 1e6)
        return q, wd

    def rhs(self, dt, mob_w, mob_o, mob_g, q_wells, dpx, dpy, dpz, ct):
        """``_build_pressure_rhs`` (simulation.py:1582-1620)."""
        comp = (self.pv * ct / dt) * self.p
        Qg = np.zeros((self.nx, self.ny, self.nz))
        if self.dz > 0 and self.nz > 1:
            Mw, Mo, Mg = self.shape(mob_w), self.shape(mob_o), self.shape(mob_g)
            rw, ro, rg = (self.shape(r) for r in self.densities(self.p))
            up = dpz > 0
            mwz = np.where(up, Mw[:, :, :-1], Mw[:, :, 1:])
            moz = np.where(up, Mo[:, :, :-1], Mo[:, :, 1:])
            mgz = np.where(up, Mg[:, :, :-1], Mg[:, :, 1:])
            rwz = np.where(up, rw[:, :, :-1], rw[:, :, 1:])
            roz = np.where(up, ro[:, :, :-1], ro[:, :, 1:])
            rgz = np.where(up, rg[:, :, :-1], rg[:, :, 1:])
            gf = self.Tz * G * self.dz * (mwz * rwz + moz * roz + mgz * rgz)
            Qg[:, :, :-1] -= gf
            Qg[:, :, 1:] += gf
        Qpc = np.zeros((self.nx, self.ny, self.nz))
        if self.pc_scale > 0:
            pc = self.shape(self.capillary(self.sw))
            Mo = self.shape(mob_o)
            mox = np.where(dpx > 0, Mo[:-1], Mo[1:])
            moy = np.where(dpy > 0, Mo[:, :-1], Mo[:, 1:])
            moz = np.where(dpz > 0, Mo[:, :, :-1], Mo[:, :, 1:])
            fx = self.Tx * mox * (pc[1:] - pc[:-1])
            fy = self.Ty * moy * (pc[:, 1:] - pc[:, :-1])
            fz = self.Tz * moz * (pc[:, :, 1:] - pc[:, :, :-1])
            Qpc[1:] += fx
            Qpc[:-1] -= fx
            Qpc[:, 1:] += fy
            Qpc[:, :-1] -= fy
            Qpc[:, :, 1:] += fz
            Qpc[:, :, :-1] -= fz
        return comp + q_wells + Qg.ravel() + Qpc.ravel()

    # -------------------------------------------------------- saturation step
    def saturation(self, p_new, dt):
        """``_impes_saturation_step`` (simulation.py:968-1544); updates sw/sg/so."""
        eps_pv = 1e-12
        nx, ny, nz = self.nx, self.ny, self.nz
        sw_old, sg_old = self.sw, self.sg
        kro, krw, krg = self.relperms(sw_old, sg_old)
        mu_o, mu_w, mu_g = self.viscosities(p_new)
        mob_w = krw / mu_w
        mob_o = kro / mu_o
        mob_g = krg / mu_g
        mob_t = mob_w + mob_o + mob_g
        P = self.shape(p_new)
        Mw, Mg = self.shape(mob_w), self.shape(mob_g)
        dpx = P[:-1] - P[1:]
        dpy = P[:, :-1] - P[:, 1:]
        dpz = P[:, :, :-1] - P[:, :, 1:]
        mwx = np.where(dpx > 0, Mw[:-1], Mw[1:]); mwy = np.where(dpy > 0, Mw[:, :-1], Mw[:, 1:])
        mwz = np.where(dpz > 0, Mw[:, :, :-1], Mw[:, :, 1:])
        mgx = np.where(dpx > 0, Mg[:-1], Mg[1:]); mgy = np.where(dpy > 0, Mg[:, :-1], Mg[:, 1:])
        mgz = np.where(dpz > 0, Mg[:, :, :-1], Mg[:, :, 1:])
        rho_w, rho_o, rho_g = self.densities(p_new)
        if self.dz > 0 and nz > 1:
            rw, rg = self.shape(rho_w), self.shape(rho_g)
            rwa = 0.5 * (rw[:, :, :-1] + rw[:, :, 1:])
            rga = 0.5 * (rg[:, :, :-1] + rg[:, :, 1:])
            pot_w_z = dpz + G * rwa * self.dz
            pot_g_z = dpz + G * rga * self.dz
        else:
            pot_w_z = dpz
            pot_g_z = dpz
        fwx = self.Tx * mwx * dpx; fwy = self.Ty * mwy * dpy; fwz = self.Tz * mwz * pot_w_z
        if self.pc_og_scale > 0:
            pcog = self.shape(self.capillary_og(sg_old))
            fgx = self.Tx * mgx * (dpx - (pcog[1:] - pcog[:-1]))
            fgy = self.Ty * mgy * (dpy - (pcog[:, 1:] - pcog[:, :-1]))
            fgz = self.Tz * mgz * (pot_g_z - (pcog[:, :, 1:] - pcog[:, :, :-1]))
        else:
            fgx = self.Tx * mgx * dpx; fgy = self.Ty * mgy * dpy; fgz = self.Tz * mgz * pot_g_z

        def div(fx, fy, fz):
            d = np.zeros((nx, ny, nz))
            d[:-1] += fx; d[1:] -= fx
            d[:, :-1] += fy; d[:, 1:] -= fy
            d[:, :, :-1] += fz; d[:, :, 1:] -= fz
            return d.ravel()

        div_w, div_g = div(fwx, fwy, fwz), div(fgx, fgy, fgz)
        fw = mob_w / (mob_t + 1e-10)
        fg = mob_g / (mob_t + 1e-10)
        fo = mob_o / (mob_t + 1e-10)
        q_w, q_g, q_o = self.well_sources(p_new, dt, mob_t, fw, fg, fo)

        dSw = (dt / self.pv) * (q_w - div_w)
        dSg = (dt / self.pv) * (q_g - div_g)
        max_dS = self.sim_params.get("max_saturation_change", 0.05)
        so_r, sw_cr, sg_cr, eps = float(self.so_r), float(self.sw_cr), float(self.sg_cr), 1e-12
        sw_up = np.maximum(1.0 - so_r - sg_old - sw_old, 0.0)
        sw_dn = np.maximum(sw_old - sw_cr, 0.0)
        sg_up = np.maximum(1.0 - so_r - sw_old - sg_old, 0.0)
        sg_dn = np.maximum(sg_old - sg_cr, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            rat_w = np.where(dSw > 0, dSw / np.maximum(sw_up, eps), (-dSw) / np.maximum(sw_dn, eps))
            rat_g = np.where(dSg > 0, dSg / np.maximum(sg_up, eps), (-dSg) / np.maximum(sg_dn, eps))
            rat_lim = np.maximum(np.abs(dSw) / max_dS, np.abs(dSg) / max_dS)
        rat = np.maximum(np.maximum(rat_w, rat_g), rat_lim)
        rat_max = rat.max()
        if not np.isfinite(rat_max):        # torch.nan_to_num(nan=0, posinf=0, neginf=0)
            rat_max = 0.0
        n_sub = int(math.ceil(rat_max))
        n_sub = max(n_sub, 1)
        n_sub = min(n_sub, int(self.sim_params.get("max_substeps", 20)))
        self.last_substeps = n_sub
        dsw_sub, dsg_sub = dSw / n_sub, dSg / n_sub
        sw, sg = sw_old, sg_old
        for _ in range(n_sub):
            sw = sw + dsw_sub
            sg = sg + dsg_sub
            sw = np.minimum(np.maximum(sw, sw_cr), 1.0 - so_r - sg)
            sg = np.minimum(np.maximum(sg, sg_cr), 1.0 - so_r - sw)
            if self.pvt is not None:
                self._component_substep(p_new, dt, n_sub, sw, sg)
        dsw_eff, dsg_eff = sw - sw_old, sg - sg_old
        mw = dsw_eff * self.pv * rho_w
        mg = dsg_eff * self.pv * rho_g
        mo = (-(dsw_eff + dsg_eff)) * self.pv * rho_o
        for ph, m in (("water", mw), ("gas", mg), ("oil", mo)):
            self.mass_balance[ph]["in"] += float(np.maximum(m, 0).sum())
            self.mass_balance[ph]["out"] += float((-np.minimum(m, 0)).sum())
        cb = self.component_balance
        cb["oil"]["accum"] = cb["oil"]["in"] - cb["oil"]["out"]
        cb["gas"]["accum"] = cb["gas"]["in"] - cb["gas"]["out"]
        self.sw, self.sg = sw, sg
        self.so = (1.0 - sw) - sg
        return n_sub

    def _pvt_cell(self, p_new, c):
        vals = {k: float(self.ev(p_new[c:c + 1], k)[0]) for k in ("Bo", "Bw", "Bg", "Rs", "Rv")}
        return vals["Bo"], vals["Bw"], vals["Bg"], vals["Rs"], vals["Rv"]

    def well_sources(self, p_new, dt, mob_t, fw, fg, fo):
        """Per-well sources of the saturation step (simulation.py:1051-1347)."""
        N = self.N
        q_w, q_g, q_o = np.zeros(N), np.zeros(N), np.zeros(N)
        cb = self.component_balance
        sw_old, sg_old = self.sw, self.sg
        rate_scale = float(self.sim_params.get("global_rate_scale", 1.0))
        so_r, sw_min, sg_min = float(self.so_r), float(self.sw_cr), float(self.sg_cr)
        for w in self.wells:
            if w.i >= self.nx or w.j >= self.ny or w.k >= self.nz:
                continue
            c = self.cell(w)
            pv_c = float(self.pv[c])
            sw, sg = float(sw_old[c]), float(sg_old[c])
            fo_, fw_, fg_ = float(fo[c]), float(fw[c]), float(fg[c])
            if w.control_type == "rate":
                q_base = (w.control_value * rate_scale) / 86400.0
                if w.type == "injector" and w.rate_type == "surface" and self.pvt is not None:
                    Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
                    q_total = q_base * (Bg if w.injected_phase == "gas" else Bw)
                else:
                    q_total = q_base
                q_total *= (1 if w.type == "injector" else -1)
                if w.type == "injector":
                    if w.injected_phase == "gas":
                        sg_up = max(0.0, (1.0 - so_r - sw) - sg)
                        dS = (dt / max(pv_c, 1e-12)) * q_total
                        alpha = 1.0
                        if dS > 0.0:
                            alpha = min(alpha, sg_up / max(dS, 1e-12))
                        else:
                            alpha = min(alpha, (sg - sg_min) / max(abs(dS), 1e-12))
                        q_total *= max(0.0, min(1.0, alpha))
                        q_g[c] += q_total
                        if self.pvt is not None:
                            Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
                            qg_surf = max(q_total, 0.0) / max(Bg, 1e-12) * 86400.0
                            scale = float(dt / 86400.0)
                            cb["gas"]["in"] += float(qg_surf * scale)
                            cb["oil"]["in"] += float(Rv * qg_surf * scale)
                    else:
                        sw_up = max(0.0, (1.0 - so_r - sg) - sw)
                        dS = (dt / max(pv_c, 1e-12)) * q_total
                        alpha = 1.0
                        if dS > 0.0:
                            alpha = min(alpha, sw_up / max(dS, 1e-12))
                        else:
                            alpha = min(alpha, (sw - sw_min) / max(abs(dS), 1e-12))
                        q_total *= max(0.0, min(1.0, alpha))
                        q_w[c] += q_total
                    continue
                # producers at rate
                if self.pvt is not None:
                    Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
                    if w.rate_type == "surface":
                        sp_ = (w.surface_phase or "liquid").lower()
                        if sp_ == "oil":
                            q_total = -(q_base / max(fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12), 1e-12))
                        elif sp_ == "water":
                            q_total = -(q_base * Bw) / max(fw_, 1e-8)
                        elif sp_ == "gas":
                            q_total = -(q_base / max(fg_ / max(Bg, 1e-12) + fo_ * Rs / max(Bo, 1e-12), 1e-12))
                        else:
                            q_total = -(q_base / max(fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12)
                                                     + fw_ / max(Bw, 1e-12), 1e-12))
                    sw_up = max(0.0, (1.0 - so_r - sg) - sw)
                    sw_dn = max(0.0, sw - sw_min)
                    sg_up = max(0.0, (1.0 - so_r - sw) - sg)
                    sg_dn = max(0.0, sg - sg_min)
                    dSw_w = (dt / max(pv_c, 1e-12)) * (q_total * fw_)
                    dSg_w = (dt / max(pv_c, 1e-12)) * (q_total * fg_)
                    alpha = 1.0
                    alpha = min(alpha, sw_up / max(dSw_w, 1e-12)) if dSw_w > 0.0 else min(alpha, sw_dn / max(abs(dSw_w), 1e-12))
                    alpha = min(alpha, sg_up / max(dSg_w, 1e-12)) if dSg_w > 0.0 else min(alpha, sg_dn / max(abs(dSg_w), 1e-12))
                    alpha = max(0.0, min(1.0, alpha))
                    q_total *= alpha
                    lim = w.limits or {}
                    if lim:
                        d_o = fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12)
                        d_w = fw_ / max(Bw, 1e-12)
                        d_g = fg_ / max(Bg, 1e-12) + fo_ * Rs / max(Bo, 1e-12)
                        d_l = d_o + d_w
                        cand = []
                        if "wopr" in lim and d_o > 0:
                            cand.append((lim["wopr"] / 86400.0) / d_o)
                        if "wlpr" in lim and d_w > 0:
                            cand.append((lim["wlpr"] / 86400.0) / d_w)
                        if "wgpr" in lim and d_g > 0:
                            cand.append((lim["wgpr"] / 86400.0) / d_g)
                        if "liqr" in lim and d_l > 0:
                            cand.append((lim["liqr"] / 86400.0) / d_l)
                        if cand:
                            mx = min(cand)
                            if abs(q_total) > mx:
                                q_total = -mx
                    oil_s = abs(q_total) * (fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12)) * 86400.0
                    wat_s = abs(q_total) * (fw_ / max(Bw, 1e-12)) * 86400.0
                    gas_s = abs(q_total) * (fg_ / max(Bg, 1e-12) + fo_ * Rs / max(Bo, 1e-12)) * 86400.0
                    w.last_surface_rates = {"oil": oil_s, "water": wat_s, "gas": gas_s, "liquid": oil_s + wat_s}
                    w.last_q_total = float(q_total)
                    qo_res, qg_res = float(-q_total * fo_), float(-q_total * fg_)
                    cb["oil"]["out"] += float(dt) * (max(qo_res, 0.0) / max(Bo, 1e-12) + Rv * max(qg_res, 0.0) / max(Bg, 1e-12))
                    cb["gas"]["out"] += float(dt) * (max(qg_res, 0.0) / max(Bg, 1e-12) + Rs * max(qo_res, 0.0) / max(Bo, 1e-12))
                q_w[c] += q_total * fw[c]
                q_g[c] += q_total * fg[c]
                q_o[c] += q_total * fo[c]
            elif w.control_type == "bhp":
                p_bhp = w.control_value * 1e6
                q_total = w.well_index * mob_t[c] * (p_new[c] - p_bhp)
                if w.type == "injector":
                    if w.injected_phase == "gas":
                        q_g[c] += -q_total
                        if self.pvt is not None:
                            Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
                            qg_surf = max(-q_total, 0.0) / max(Bg, 1e-12) * 86400.0
                            scale = float(dt / 86400.0)
                            cb["gas"]["in"] += float(qg_surf * scale)
                            cb["oil"]["in"] += float(Rv * qg_surf * scale)
                    else:
                        q_w[c] += -q_total
                else:
                    q_w[c] += (-q_total) * fw[c]
                    q_g[c] += (-q_total) * fg[c]
                    q_o[c] += (-q_total) * fo[c]
                    if self.pvt is not None:
                        Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
                        qabs = abs(q_total)
                        qo_res, qg_res = qabs * fo_, qabs * fg_
                        cb["oil"]["out"] += float(dt) * (qo_res / max(Bo, 1e-12) + Rv * qg_res / max(Bg, 1e-12))
                        cb["gas"]["out"] += float(dt) * (qg_res / max(Bg, 1e-12) + Rs * qo_res / max(Bo, 1e-12))
        return q_w, q_g, q_o

    def _component_substep(self, p_new, dt, n_sub, sw, sg):
        """Per-substep component balance of PVT runs (simulation.py:1396-1505)."""
        cb = self.component_balance
        rate_scale = float(self.sim_params.get("global_rate_scale", 1.0))
        dt_sub = dt / n_sub
        for w in self.wells:
            if w.i >= self.nx or w.j >= self.ny or w.k >= self.nz:
                continue
            c = self.cell(w)
            cs = slice(c, c + 1)
            Bo, Bw, Bg, Rs, Rv = self._pvt_cell(p_new, c)
            mu_w = self.ev(p_new[cs], "mu_w"); mu_o = self.ev(p_new[cs], "mu_o"); mu_g = self.ev(p_new[cs], "mu_g")
            kro, krw, krg = self.relperms(sw[cs], sg[cs])
            mw = krw / (mu_w + 1e-12); mo = kro / (mu_o + 1e-12); mg = krg / (mu_g + 1e-12)
            mt = mw + mo + mg
            fw_ = float((mw / (mt + 1e-12))[0]); fg_ = float((mg / (mt + 1e-12))[0]); fo_ = float((mo / (mt + 1e-12))[0])
            if w.control_type == "rate":
                q_base = (w.control_value * rate_scale) / 86400.0
                if w.type == "injector":
                    if w.rate_type == "surface":
                        q_sub = q_base * (Bg if w.injected_phase == "gas" else Bw)
                    else:
                        q_sub = q_base
                    if w.injected_phase == "gas":
                        qg_surf = max(q_sub, 0.0) / max(Bg, 1e-12) * 86400.0
                        cb["gas"]["in"] += float(qg_surf * (dt_sub / 86400.0))
                        cb["oil"]["in"] += float(Rv * qg_surf * (dt_sub / 86400.0))
                else:
                    if w.rate_type == "surface":
                        sp_ = (w.surface_phase or "liquid").lower()
                        if sp_ == "oil":
                            q_sub = -(q_base / max(fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12), 1e-12))
                        elif sp_ == "water":
                            q_sub = -(q_base * Bw) / max(fw_, 1e-12)
                        elif sp_ == "gas":
                            q_sub = -(q_base / max(fg_ / max(Bg, 1e-12) + fo_ * Rs / max(Bo, 1e-12), 1e-12))
                        else:
                            q_sub = -(q_base / max(fo_ / max(Bo, 1e-12) + fg_ * Rv / max(Bg, 1e-12)
                                                   + fw_ / max(Bw, 1e-12), 1e-12))
                    else:
                        q_sub = -q_base
                    qo_res, qg_res = max(-q_sub * fo_, 0.0), max(-q_sub * fg_, 0.0)
                    cb["oil"]["out"] += float(dt_sub * (qo_res / max(Bo, 1e-12) + Rv * qg_res / max(Bg, 1e-12)))
                    cb["gas"]["out"] += float(dt_sub * (qg_res / max(Bg, 1e-12) + Rs * qo_res / max(Bo, 1e-12)))
            elif w.control_type == "bhp":
                q_sub = w.well_index * float(mt[0]) * (float(p_new[c]) - w.control_value * 1e6)
                if w.type == "injector":
                    if w.injected_phase == "gas":
                        qg_surf = max(-q_sub, 0.0) / max(Bg, 1e-12) * 86400.0
                        cb["gas"]["in"] += float(qg_surf * (dt_sub / 86400.0))
                        cb["oil"]["in"] += float(Rv * qg_surf * (dt_sub / 86400.0))
                else:
                    qabs = abs(q_sub)
                    cb["oil"]["out"] += float(dt_sub * (qabs * fo_ / max(Bo, 1e-12) + Rv * (qabs * fg_) / max(Bg, 1e-12)))
                    cb["gas"]["out"] += float(dt_sub * (qabs * fg_ / max(Bg, 1e-12) + Rs * (qabs * fo_) / max(Bo, 1e-12)))

    # ------------------------------------------------------------------- step
    def step(self, dt, solve="direct"):
        """One ``_impes_step`` attempt (simulation.py:822-865): pressure, then saturation.

        ``solve`` is "direct", "cg" (the reference's Jacobi-PCG with its retry,
        simulation.py:931-966; returns (None, 0) when both attempts miss) or a
        callable (A, b) -> x."""
        A, b, _ = self.assemble(dt)
        if solve == "direct":
            p_new = spla.spsolve(A.tocsc(), b)
        elif solve == "cg":
            tol = float(self.sim_params.get("cg_tolerance", 1e-6))
            it = int(self.sim_params.get("cg_max_iter", 500))
            diag = A.diagonal()
            p_new, ok, _ = pcg_solve(A, b, diag, tol, it)
            if not ok:
                p_new, ok, _ = pcg_solve(A, b, diag, tol * 10.0, it * 4)
            if not ok:
                return None, 0
        else:
            p_new = solve(A, b)
        p_new = np.asarray(p_new, dtype=np.float64)
        self.p = p_new
        n_sub = self.saturation(p_new, dt)
        return p_new, n_sub


def pcg_solve(A, b, m_diag, tol=1e-6, max_iter=500):
    """``_solve_pressure_cg_pytorch`` (simulation.py:1662-1697): Jacobi-preconditioned
    CG from x = 0, stopping when sqrt(r . M^-1 r) < tol (absolute).  Returns
    (x, converged, iterations)."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    r = b - A @ x
    z = r / m_diag
    p = z.copy()
    rs_old = float(r @ z)
    if rs_old < 1e-10:
        return x, True, 0
    for i in range(max_iter):
        Ap = A @ p
        alpha = rs_old / float(p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        z = r / m_diag
        rs_new = float(r @ z)
        if math.sqrt(rs_new) < tol:
            return x, True, i + 1
        p = z + (rs_new / rs_old) * p
        rs_old = rs_new
    return x, False, max_iter
