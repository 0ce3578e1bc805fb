"""Seeded synthetic workloads for the IMPES path.

Each builder returns ``(cfg, fields)``: ``cfg`` is a config dict in the
reference's JSON schema (sections ``reservoir``, ``fluid``, ``wells``,
``simulation``) and ``fields`` holds the heterogeneous rock the schema cannot
express -- ``kx, ky, kz`` in m^2 and ``poro``, as float64 arrays shaped
``(nx, ny, nz)`` (flat index ``(i*ny + j)*nz + k``) -- plus, for black-oil
cases, ``pvt`` (a table dict in the reference's PVT JSON layout).

Workloads (sizes as named):

* ``two_phase_2d``      64x64x1, dx=dy=10 m, dz=5 m, oil-water, Corey, 100 x 1 d
* ``black_oil_5spot``   100x100x20, 20x20x2 m, 20-row PVT, Stone II, gravity,
                        capillarity, 4 rate injectors + 1 BHP producer, 50 x 5 d
* ``gas_injection_1m``  200x200x25 = 1e6 cells, correlated log-normal k,
                        9 surface-rate gas injectors + 16 BHP producers, 20 x 2 d
* ``three_phase``       16x16x3 oil-water-gas without PVT (constant
                        compressibilities), initial free gas above Sgc, a gas
                        and a water injector, two rate producers, 10 x 1 d
* ``adjoint_case``      64x64x8 with the two-phase fluids, 50 x 2 d
* ``ensemble``          64 uneven realisations (nx, ny in {32..128}, nz in {4,8,16})

All randomness comes from ``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import math

import numpy as np

MD = 9.869233e-16   # mD -> m^2, as the reference converts (reservoir.py:35)


def _lognormal(rng, shape, mean_md, sigma):
    return np.exp(math.log(mean_md) + sigma * rng.standard_normal(shape)) * MD


def pvt_table_black_oil(rows: int = 20, p_lo: float = 5.0, p_hi: float = 40.0,
                        bo_increasing: bool = False, rv_max: float = 0.0) -> dict:
    """Monotone synthetic black-oil table over ``p_lo..p_hi`` MPa.

    Bo spans 1.1..1.3, Rs 0 -> 150, mu_o 3 -> 1.5 cP, mu_g 0.012 -> 0.025 cP
    (all linear in p); Bg 0.02 -> 0.003 as ``a/p + b`` through both end points;
    water is slightly compressible (Bw 1.02 -> 1.00) with mu_w 0.5 cP.  Rv
    (vaporised oil, ``Rv_m3m3``) rises linearly from 0 to ``rv_max``; with the
    default 0 the column is left out, as the reference's loader allows.

    Bo decreases with pressure by default (1.3 at p_lo to 1.1 at p_hi).  The
    reference's total compressibility c_o = -(1/Bo) dBo/dP (fluid.py:190-222) has
    no dissolved-gas term, so a Bo that grows with pressure (``bo_increasing``)
    makes c_t negative and the pressure matrix indefinite.
    """
    p = np.linspace(p_lo, p_hi, rows)
    t = (p - p_lo) / (p_hi - p_lo)
    a = (0.02 - 0.003) / (1.0 / p_lo - 1.0 / p_hi)
    b = 0.02 - a / p_lo
    return {
        "pressure_MPa": p.tolist(),
        "Bo": ((1.1 + 0.2 * t) if bo_increasing else (1.3 - 0.2 * t)).tolist(),
        "Bw": (1.02 - 0.02 * t).tolist(),
        "Bg": (a / p + b).tolist(),
        "mu_o_cP": (3.0 - 1.5 * t).tolist(),
        "mu_w_cP": np.full(rows, 0.5).tolist(),
        "mu_g_cP": (0.012 + 0.013 * t).tolist(),
        "Rs_m3m3": (150.0 * t).tolist(),
        **({"Rv_m3m3": (rv_max * t).tolist()} if rv_max > 0.0 else {}),
    }


def _two_phase_fluid(p_mpa=20.0):
    # 1e-5 1/bar = 1e-4 1/MPa; c_gas = 0 makes the reference's (co+cw+cg+cr)/3 equal 1e-4/MPa
    return {
        "pressure": p_mpa, "s_w": 0.2, "s_g": 0.0,
        "mu_oil": 5.0, "mu_water": 1.0,
        "c_oil": 1e-4, "c_water": 1e-4, "c_rock": 1e-4, "c_gas": 0.0,
        "relative_permeability": {"model": "corey", "nw": 2.0, "no": 2.0, "sw_cr": 0.2, "so_r": 0.2},
        "capillary_pressure": {"pc_scale": 0.0},
    }


def _sim(dt_days, steps, solver="gmres_amg", tol=1e-6, max_cycles=40):
    return {
        "solver_type": "impes", "time_step_days": dt_days, "total_time_days": dt_days * steps,
        "pressure_solver": solver,
        "amg": {"tol": tol, "max_cycles": max_cycles, "theta": 0.25, "max_levels": 10,
                "coarsest_size": 200, "device": "auto"},
    }


def two_phase_2d(seed: int = 0, nx: int = 64, ny: int = 64, nz: int = 1, steps: int = 100,
                 sigma: float = 0.5, dt_days: float = 1.0):
    """64x64x1 oil-water: ln k ~ N(ln 100 mD, sigma^2) i.i.d., phi ~ U[0.18, 0.22]."""
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz)
    k = _lognormal(rng, shape, 100.0, sigma)
    poro = 0.18 + 0.04 * rng.random(shape)
    cfg = {
        "reservoir": {"dimensions": [nx, ny, nz], "grid_size": [10.0, 10.0, 5.0], "porosity": 0.2,
                      "permeability": 100.0, "k_vertical_fraction": 1.0, "c_rock": 1e-4},
        "fluid": _two_phase_fluid(),
        "wells": [
            {"name": "INJ", "type": "injector", "i": 0, "j": 0, "k": 0, "radius": 0.1,
             "control_type": "rate", "control_value": 50.0, "injected_phase": "water"},
            {"name": "PROD", "type": "producer", "i": nx - 1, "j": ny - 1, "k": 0, "radius": 0.1,
             "control_type": "bhp", "control_value": 15.0},
        ],
        "simulation": _sim(dt_days, steps),
    }
    return cfg, {"kx": k, "ky": k.copy(), "kz": k.copy(), "poro": poro}


def three_phase(seed: int = 6, nx: int = 16, ny: int = 16, nz: int = 3, steps: int = 10,
                dt_days: float = 1.0, rate: float = 10.0):
    """Three phases without PVT: ln k ~ N(ln 120 mD, 0.6^2) i.i.d., kz = 0.1 kx,
    phi ~ U[0.2, 0.25]; Sw = 0.2, Sg = 0.04 (Sgc 0.02) at 22 MPa; c_gas = 1e-3
    1/MPa; Corey with ng = 2.5; a gas and a water injector and two producers,
    all rate-controlled at ``rate`` m3/d, in the middle layer.

    The producers are rate wells on purpose.  A BHP producer's cell sits at the
    well pressure to within rounding, so its saturation-step rate
    WI*lambda*(p - p_bhp) (simulation.py:1297) is rounding noise; with mobile gas
    that noise decides the trajectory within a few steps (the reference's own
    run of this case with BHP producers reaches Sw = -0.6 at the fifth step).
    Near the substep cap of 20 the explicit update is fragile too: on the
    reference's configs/gas_injection_3phase.json, run in float64, a gas
    injector's cell passes Sg > 1 - Sor - Swc at the third step and the clamp
    order (Sw to [Swc, 1 - Sor - Sg] first) takes Sw below Swc."""
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz)
    k = _lognormal(rng, shape, 120.0, 0.6)
    poro = 0.2 + 0.05 * rng.random(shape)
    km = nz // 2
    cfg = {
        "reservoir": {"dimensions": [nx, ny, nz], "grid_size": [10.0, 10.0, 5.0], "porosity": 0.22,
                      "permeability": 120.0, "k_vertical_fraction": 0.1, "c_rock": 1e-5},
        "fluid": {
            "pressure": 22.0, "s_w": 0.2, "s_g": 0.04,
            "mu_oil": 1.8, "mu_water": 0.5, "mu_gas": 0.02,
            "rho_oil": 840.0, "rho_water": 1000.0, "rho_gas": 1.1,
            "c_oil": 1e-5, "c_water": 5e-6, "c_gas": 1e-3, "c_rock": 1e-5,
            "relative_permeability": {"nw": 2.0, "no": 2.0, "ng": 2.5, "sw_cr": 0.15, "so_r": 0.2,
                                      "sg_cr": 0.02},
            "capillary_pressure": {"pc_scale": 0.0},
        },
        "wells": [
            {"name": "GI", "type": "injector", "i": 2, "j": ny // 2, "k": km, "radius": 0.1,
             "control_type": "rate", "control_value": rate, "injected_phase": "gas"},
            {"name": "WI", "type": "injector", "i": nx - 3, "j": ny // 2, "k": km, "radius": 0.1,
             "control_type": "rate", "control_value": rate, "injected_phase": "water"},
            {"name": "P1", "type": "producer", "i": nx // 2, "j": 3, "k": km, "radius": 0.1,
             "control_type": "rate", "control_value": rate},
            {"name": "P2", "type": "producer", "i": nx // 2, "j": ny - 4, "k": km, "radius": 0.1,
             "control_type": "rate", "control_value": rate},
        ],
        "simulation": _sim(dt_days, steps),
    }
    return cfg, {"kx": k, "ky": k.copy(), "kz": 0.1 * k, "poro": poro}


def _black_oil_fluid(pvt):
    return {
        "pressure": 25.0, "s_w": 0.2, "s_g": 0.0,
        "rho_oil": 850.0, "rho_water": 1000.0, "rho_gas": 1.0,
        "c_rock": 1e-4,
        "pvt": {"table": pvt},
        "relative_permeability": {"model": "stone2", "nw": 2.0, "no": 2.0, "ng": 2.5,
                                  "sw_cr": 0.2, "so_r": 0.2, "sg_cr": 0.0},
        # Brooks-Corey entry 0.5 bar, lambda = 2 -> pc_scale 5e4 Pa, exponent 1/lambda
        "capillary_pressure": {"pc_scale": 5.0e4, "pc_exponent": 0.5},
    }


def black_oil_5spot(seed: int = 1, nx: int = 100, ny: int = 100, nz: int = 20, steps: int = 50,
                    inj_rate: float = 200.0, dt_days: float = 5.0, bo_increasing: bool = False):
    """Three-phase black oil: ln kx ~ N(ln 200 mD, 0.8^2) per cell, ky=kx, kz=0.1 kx."""
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz)
    kx = _lognormal(rng, shape, 200.0, 0.8)
    poro = 0.15 + 0.10 * rng.random(shape)
    pvt = pvt_table_black_oil(bo_increasing=bo_increasing)
    km = nz // 2
    inj = [(0, 0), (nx - 1, 0), (0, ny - 1), (nx - 1, ny - 1)]
    wells = [{"name": f"INJ{n}", "type": "injector", "i": i, "j": j, "k": km, "radius": 0.1,
              "control_type": "rate", "control_value": inj_rate, "injected_phase": "water"}
             for n, (i, j) in enumerate(inj)]
    wells.append({"name": "PROD", "type": "producer", "i": nx // 2, "j": ny // 2, "k": km,
                  "radius": 0.1, "control_type": "bhp", "control_value": 12.0})
    cfg = {
        "reservoir": {"dimensions": [nx, ny, nz], "grid_size": [20.0, 20.0, 2.0], "porosity": 0.2,
                      "permeability": 200.0, "k_vertical_fraction": 0.1, "c_rock": 1e-4},
        "fluid": _black_oil_fluid(pvt),
        "wells": wells,
        "simulation": _sim(dt_days, steps),
    }
    return cfg, {"kx": kx, "ky": kx.copy(), "kz": 0.1 * kx, "poro": poro, "pvt": pvt}


def _gaussian_smooth(z, sigma=2.5, radius=5):
    """Separable Gaussian filter (reflect boundary), then rescaled to unit variance."""
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    w = np.exp(-0.5 * (x / sigma) ** 2)
    w /= w.sum()
    out = z
    for ax in range(z.ndim):
        pad = [(0, 0)] * z.ndim
        pad[ax] = (radius, radius)
        zp = np.pad(out, pad, mode="reflect")
        acc = np.zeros_like(out)
        for o, wo in enumerate(w):
            sl = [slice(None)] * z.ndim
            sl[ax] = slice(o, o + out.shape[ax])
            acc += wo * zp[tuple(sl)]
        out = acc
    out = out - out.mean()
    return out / out.std()


def gas_injection_1m(seed: int = 2, nx: int = 200, ny: int = 200, nz: int = 25, steps: int = 20,
                     dt_days: float = 2.0, gas_rate: float = 2.0e5, n_inj_side: int = 3,
                     n_prod_side: int = 4, surface_units: bool = False, bo_increasing: bool = False,
                     rate_scale: float = 0.05):
    """Gas-injection stress case: ln k ~ N(ln 150 mD, 1.0^2) Gaussian-correlated (radius 5).

    ``gas_rate`` is in sm3/d.  By default each injector is given the equivalent
    reservoir rate, gas_rate * Bg(initial pressure), as a ``rate_type:
    "reservoir"`` well: the reference's pressure step injects a surface-rate
    well's number unconverted, as reservoir m3/s (simulation.py:1626-1634, while
    the saturation step converts it with Bg at :1061-1064), which at 2e5 sm3/d
    drives the explicit saturation update out of range.  ``surface_units=True``
    keeps the literal surface-rate wells.  ``rate_scale`` is the simulation's
    ``global_rate_scale``.
    """
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz)
    z = _gaussian_smooth(rng.standard_normal(shape))
    kx = np.exp(math.log(150.0) + 1.0 * z) * MD
    poro = 0.15 + 0.10 * rng.random(shape)
    pvt = pvt_table_black_oil(bo_increasing=bo_increasing)
    p0 = 25.0
    bg0 = float(np.interp(p0, pvt["pressure_MPa"], pvt["Bg"]))
    km = nz // 2
    wells = []
    for a in range(n_inj_side):
        for b in range(n_inj_side):
            i = int((a + 0.5) * nx / n_inj_side); j = int((b + 0.5) * ny / n_inj_side)
            if surface_units:
                wells.append({"name": f"GI{a}{b}", "type": "injector", "i": i, "j": j, "k": km,
                              "radius": 0.1, "control_type": "rate", "control_value": gas_rate,
                              "injected_phase": "gas", "rate_type": "surface"})
            else:
                wells.append({"name": f"GI{a}{b}", "type": "injector", "i": i, "j": j, "k": km,
                              "radius": 0.1, "control_type": "rate", "control_value": gas_rate * bg0,
                              "injected_phase": "gas", "rate_type": "reservoir"})
    for a in range(n_prod_side):
        for b in range(n_prod_side):
            i = int(a * (nx - 1) / max(n_prod_side - 1, 1)); j = int(b * (ny - 1) / max(n_prod_side - 1, 1))
            wells.append({"name": f"P{a}{b}", "type": "producer", "i": i, "j": j, "k": km,
                          "radius": 0.1, "control_type": "bhp", "control_value": 15.0})
    fluid = _black_oil_fluid(pvt)
    sim = _sim(dt_days, steps)
    # the reference's own AMG settings for its million-cell case
    # (configs/mega_3phase_million.json:19-25; docs/PERFORMANCE.md:44-46)
    sim["amg"].update({"theta": 0.2, "max_levels": 20, "coarsest_size": 120})
    # and its rate scale and substep cap (configs/mega_3phase_million.json:13-14): at the
    # unscaled 2e5 sm3/d an injector cell takes ~20 pore volumes per 2-day step and the
    # explicit update leaves [0, 1] (Sw -8, Sg 9 after four steps, reference semantics)
    sim.update({"global_rate_scale": rate_scale, "max_substeps": 20})
    cfg = {
        "reservoir": {"dimensions": [nx, ny, nz], "grid_size": [20.0, 20.0, 2.0], "porosity": 0.2,
                      "permeability": 150.0, "k_vertical_fraction": 0.1, "c_rock": 1e-4},
        "fluid": fluid,
        "wells": wells,
        "simulation": sim,
    }
    return cfg, {"kx": kx, "ky": kx.copy(), "kz": 0.1 * kx, "poro": poro, "pvt": pvt}


def adjoint_case(seed: int = 3, nx: int = 64, ny: int = 64, nz: int = 8, steps: int = 50,
                 dt_days: float = 2.0, sigma: float = 0.7):
    """64x64x8 oil-water with the two-phase fluids and corner wells."""
    return two_phase_2d(seed=seed, nx=nx, ny=ny, nz=nz, steps=steps, sigma=sigma, dt_days=dt_days)


def ensemble(seed: int = 4, members: int = 64, steps: int = 30):
    """Uneven realisations: nx, ny in {32,48,64,96,128}, nz in {4,8,16}, sigma in [0.3, 1.2]."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(members):
        nx, ny = (int(v) for v in rng.choice([32, 48, 64, 96, 128], size=2))
        nz = int(rng.choice([4, 8, 16]))
        sig = float(rng.uniform(0.3, 1.2))
        out.append(two_phase_2d(seed=int(rng.integers(1 << 30)), nx=nx, ny=ny, nz=nz, steps=steps,
                                sigma=sig, dt_days=1.0))
    return out


WORKLOADS = {
    "two_phase_2d": two_phase_2d,
    "black_oil_5spot": black_oil_5spot,
    "gas_injection_1m": gas_injection_1m,
    "adjoint_case": adjoint_case,
}
