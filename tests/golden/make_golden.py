"""Generate the golden fixtures by running the reference itself (build container only).

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT [--pcg-only | --three-phase-only |
                                                        --wells-only | --amg-3d-only | --configs-only |
                                                        --adjoint-only]

REFERENCE_ROOT is a checkout of researchim-ai/oil-simulator-py (the directory
holding ``src/``); it may instead be given in the environment variable
OIL_SIMULATOR_REFERENCE.  There is no default.
The reference is imported unmodified; the harness only
  * puts a placeholder ``matplotlib`` first on sys.path (plotting is unused here),
  * sets ``torch.set_default_dtype(torch.float64)`` before building objects,
  * overwrites ``Reservoir.permeability_{x,y,z}``, ``porosity`` and
    ``porous_volume`` with the seeded fields before ``Simulator()`` is built,
  * replaces ``Fluid._eval_pvt``'s float32 cast with float64 (same ``np.interp``),
  * replaces ``solver.pressure_amg.amg_solve`` by a direct ``spsolve`` of the
    reference's own assembled (A, b), recording both (the trajectory oracle),
  * feeds ``torch.rand`` the deterministic C/F tie-break vector while
    ``ClassicalAMG`` builds its hierarchy.
Outputs go to ``tests/golden/*.npz``.  The fixtures hold their own inputs
(config JSON, rock fields) so tests never need the reference.
"""
from __future__ import annotations

import contextlib
import io
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
_ARGS = [a for a in sys.argv[1:] if not a.startswith("--")]
REF = _ARGS[0] if _ARGS else os.environ.get("OIL_SIMULATOR_REFERENCE", "")
if not REF or not os.path.isdir(os.path.join(REF, "src", "simulator")):
    sys.stderr.write(__doc__ + "\nerror: REFERENCE_ROOT (or OIL_SIMULATOR_REFERENCE) must name the "
                     "reference checkout\n")
    sys.exit(2)
sys.path[:0] = [os.path.join(HERE, "_stubs"), os.path.join(REF, "src"), REPO]

import torch  # noqa: E402
import scipy.sparse as sp  # noqa: E402
import scipy.sparse.linalg as spla  # noqa: E402

torch.set_default_dtype(torch.float64)
torch.set_num_threads(4)

from simulator.reservoir import Reservoir  # noqa: E402
from simulator.fluid import Fluid  # noqa: E402
from simulator.well import WellManager  # noqa: E402
from simulator.simulation import Simulator  # noqa: E402
import solver.pressure_amg as pamg  # noqa: E402
from solver.classical_amg import ClassicalAMG  # noqa: E402

from oracle.amg import tiebreak  # noqa: E402  (the shared tie-break definition)


def _load_scenarios():
    # the input generator, loaded by path: putting the package directory on
    # sys.path would shadow the reference's namespace package ``solver``
    import importlib.util
    path = os.path.join(REPO, "oil-simulator-py_b200", "impes_b200", "scenarios.py")
    spec = importlib.util.spec_from_file_location("scenarios_for_fixtures", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


scenarios = _load_scenarios()


def _eval_pvt64(self, p_tensor, key):
    p_mpa = (p_tensor.detach().to("cpu").numpy() / 1e6).astype(np.float64)
    vals = self.pvt.eval(p_mpa)[key]
    return torch.from_numpy(vals).to(self.device, dtype=torch.float64).reshape(self.dimensions)


Fluid._eval_pvt = _eval_pvt64


def build_reference(cfg, fields, tmpdir):
    cfg = json.loads(json.dumps(cfg))
    fc = cfg["fluid"]
    if isinstance(fc.get("pvt"), dict) and "table" in fc["pvt"]:
        path = os.path.join(tmpdir, "pvt.json")
        with open(path, "w") as f:
            json.dump(fc["pvt"]["table"], f)
        fc.pop("pvt")
        fc["pvt_path"] = path
    sim_cfg = dict(cfg["simulation"])
    sim_cfg["pressure_solver"] = "amg"
    dev = torch.device("cpu")
    with contextlib.redirect_stdout(io.StringIO()):
        res = Reservoir(cfg["reservoir"], dev)
        res.permeability_x = torch.from_numpy(np.ascontiguousarray(fields["kx"]))
        res.permeability_y = torch.from_numpy(np.ascontiguousarray(fields["ky"]))
        res.permeability_z = torch.from_numpy(np.ascontiguousarray(fields["kz"]))
        res.porosity = torch.from_numpy(np.ascontiguousarray(fields["poro"]))
        res.porous_volume = res.cell_volume * res.porosity
        wm = WellManager(cfg["wells"], res)
        fl = Fluid(fc, res, dev)
        sim = Simulator(res, fl, wm, sim_cfg, dev)
    return sim, fl, wm


def fields_digest(fields):
    """sha256 of the rock fields (kx, ky, kz, poro as float64 C-order bytes)."""
    import hashlib
    h = hashlib.sha256()
    for k in ("kx", "ky", "kz", "poro"):
        h.update(np.ascontiguousarray(fields[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def run_trajectory(name, cfg, fields, steps, dt_days, solver="direct", full_at=None, n_samples=0,
                   keep_systems=None, generator=None):
    """The reference's trajectory with amg_solve replaced by a direct solve of its
    own (A, b); with solver="cg" the reference's own Jacobi-PCG path runs
    unpatched (pressure_solver "cg").

    Long runs are stored compactly: ``full_at`` lists the (1-based) steps whose
    whole p/sw/sg fields are kept (None: every step), ``n_samples`` cells drawn
    with a fixed seed are kept at every step (``sample_idx``, ``p_s``, ``sw_s``,
    ``sg_s``), and only the first ``keep_systems`` assembled systems are kept
    (None: all).  With ``generator`` = (scenario function name, keyword
    arguments) the rock fields and the recorded systems are left out: tests
    rebuild the fields with that scenario call and check them against the
    stored ``fields_sha256``."""
    rec = {"A": [], "b": []}

    def direct(A, b, **kw):
        A = A.coalesce().to_sparse_csr() if A.layout == torch.sparse_coo else A
        crow, col, val = A.crow_indices().numpy(), A.col_indices().numpy(), A.values().numpy()
        if keep_systems is None or len(rec["b"]) < keep_systems:
            rec["A"].append((crow.copy(), col.copy(), val.copy()))
            rec["b"].append(b.numpy().copy())
        else:
            rec["b"].append(None)
        M = sp.csr_matrix((val, col, crow), shape=A.shape)
        return torch.from_numpy(spla.spsolve(M.tocsc(), b.numpy()))

    pamg.amg_solve = direct
    if solver == "cg":
        cfg = json.loads(json.dumps(cfg))
        cfg["simulation"]["pressure_solver"] = "cg"
        orig = Simulator._build_pressure_matrix_vectorized

        def record(self, *a, **kw):
            A, A_diag = orig(self, *a, **kw)
            C = A.coalesce().to_sparse_csr()
            rec["A"].append((C.crow_indices().numpy().copy(), C.col_indices().numpy().copy(),
                             C.values().numpy().copy()))
            return A, A_diag
        Simulator._build_pressure_matrix_vectorized = record
        orig_rhs = Simulator._build_pressure_rhs

        def record_rhs(self, *a, **kw):
            Q = orig_rhs(self, *a, **kw)
            rec["b"].append(Q.numpy().copy())
            return Q
        Simulator._build_pressure_rhs = record_rhs
    out = {}
    with tempfile.TemporaryDirectory() as td:
        sim, fl, wm = build_reference(cfg, fields, td)
        ps, sws, sgs, mbs, qs = [], [], [], [], []
        ncell = fields["kx"].size
        sidx = (np.sort(np.random.default_rng(12345).choice(ncell, size=min(n_samples, ncell),
                                                            replace=False))
                if n_samples else None)
        p_s, sw_s, sg_s = [], [], []
        for st in range(1, steps + 1):
            with contextlib.redirect_stdout(io.StringIO()):
                ok = sim.run_step(dt_days * 86400.0)
            assert ok
            p_, sw_, sg_ = (fl.pressure.numpy().ravel().copy(), fl.s_w.numpy().ravel().copy(),
                            fl.s_g.numpy().ravel().copy())
            if full_at is None or st in full_at:
                ps.append(p_); sws.append(sw_); sgs.append(sg_)
            if sidx is not None:
                p_s.append(p_[sidx]); sw_s.append(sw_[sidx]); sg_s.append(sg_[sidx])
            mb = sim.mass_balance
            cb = sim.component_balance
            mbs.append([mb[ph][io_] for ph in ("water", "oil", "gas") for io_ in ("in", "out")]
                       + [cb[c][k] for c in ("oil", "gas") for k in ("in", "out", "accum")])
            qs.append([w.last_q_total if w.last_q_total is not None else np.nan for w in wm.get_wells()])
            if steps >= 20 and st % 10 == 0:
                print(f"  {name}: step {st}/{steps}", flush=True)
        wells = [(w.cell_index_flat, w.last_q_total if w.last_q_total is not None else np.nan)
                 for w in wm.get_wells()]
    crow, col, val = rec["A"][0]
    kept_b = [b for b in rec["b"] if b is not None]
    out.update(
        cfg=json.dumps(cfg), kx=fields["kx"], ky=fields["ky"], kz=fields["kz"], poro=fields["poro"],
        dt=dt_days * 86400.0,
        A0_crow=crow.astype(np.int32), A0_col=col.astype(np.int32), A0_val=val,
        b0=rec["b"][0], b_all=np.stack(kept_b),
        A_val_all=np.stack([a[2] for a in rec["A"]]),
        p=np.stack(ps), sw=np.stack(sws), sg=np.stack(sgs), balances=np.array(mbs),
        well_cells=np.array([w[0] for w in wells], dtype=np.int64),
        well_last_q=np.array([w[1] for w in wells]),
    )
    if full_at is not None:
        out["full_at"] = np.array(sorted(full_at), dtype=np.int64)
        out["steps"] = np.array(steps)
        out["well_q_all"] = np.array(qs)
    if sidx is not None:
        out.update(sample_idx=sidx.astype(np.int64), p_s=np.stack(p_s), sw_s=np.stack(sw_s),
                   sg_s=np.stack(sg_s))
    if generator is not None:
        for k in ("kx", "ky", "kz", "poro", "A0_crow", "A0_col", "A0_val", "b0", "b_all", "A_val_all"):
            out.pop(k, None)
        out["fields_generator"] = json.dumps({"scenario": generator[0], "kwargs": generator[1]})
        out["fields_sha256"] = fields_digest(fields)
    if solver == "cg":
        Simulator._build_pressure_matrix_vectorized = orig
        Simulator._build_pressure_rhs = orig_rhs
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "N", fields["kx"].size, "steps", steps, "p range", ps[-1].min(), ps[-1].max(),
          "sw max", sws[-1].max(), "sg max", sgs[-1].max(), flush=True)
    return out


def pcg_fixture(name, traj, cases):
    """The reference's _solve_pressure_cg_pytorch (simulation.py:1662-1697) on a
    recorded first-step system, for (tol, max_iter) pairs."""
    crow, col, val = (traj["A0_crow"].astype(np.int64), traj["A0_col"].astype(np.int64),
                      traj["A0_val"])
    n = len(crow) - 1
    Acsr = torch.sparse_csr_tensor(torch.from_numpy(crow), torch.from_numpy(col), torch.from_numpy(val),
                                   size=(n, n))
    A = Acsr.to_sparse_coo().coalesce()
    diag = torch.from_numpy(sp.csr_matrix((val, col, crow), shape=(n, n)).diagonal().copy())
    b = torch.from_numpy(traj["b0"])
    out = {"A0_crow": traj["A0_crow"], "A0_col": traj["A0_col"], "A0_val": val, "b0": traj["b0"],
           "tol": np.array([c[0] for c in cases]), "max_iter": np.array([c[1] for c in cases])}
    with tempfile.TemporaryDirectory() as td:
        cfg = json.loads(str(traj["cfg"]))
        sim, _, _ = build_reference(cfg, {k: traj[k] for k in ("kx", "ky", "kz", "poro")}, td)
        for q, (tol, it) in enumerate(cases):
            x, conv = sim._solve_pressure_cg_pytorch(A, b.clone(), M_diag=diag, tol=tol, max_iter=it)
            out[f"x{q}"] = x.numpy().copy()
            out[f"converged{q}"] = np.array(bool(conv))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, [(c, bool(out[f"converged{q}"])) for q, c in enumerate(cases)])


def amg_fixture(name, traj, seed=7, coarsest=50):
    """Reference ClassicalAMG on a recorded pressure matrix, with a fixed tie-break."""
    crow, col = traj["A0_crow"].astype(np.int64), traj["A0_col"].astype(np.int64)
    A = torch.sparse_csr_tensor(torch.from_numpy(crow), torch.from_numpy(col),
                                torch.from_numpy(traj["A0_val"]), size=(len(crow) - 1,) * 2)
    calls = {"n": 0}
    real_rand = torch.rand

    def fake_rand(n, *a, **kw):
        v = torch.from_numpy(tiebreak(seed, calls["n"], int(n)))
        calls["n"] += 1
        return v

    torch.rand = fake_rand
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            amg = ClassicalAMG(A, theta=0.25, max_levels=10, coarsest_size=coarsest)
    finally:
        torch.rand = real_rand
    b = torch.from_numpy(traj["b0"])
    out = {"seed": seed, "coarsest": coarsest, "n_levels": len(amg.levels),
           "Dhalf_inv": amg.Dhalf_inv.numpy() if amg.Dhalf_inv is not None else np.zeros(0)}
    for l, lv in enumerate(amg.levels):
        Al = lv["A"]
        out[f"L{l}_A_crow"] = Al.crow_indices().numpy().astype(np.int32)
        out[f"L{l}_A_col"] = Al.col_indices().numpy().astype(np.int32)
        out[f"L{l}_A_val"] = Al.values().numpy()
        out[f"L{l}_inv_relax"] = lv["inv_relax"].numpy()
        if lv["P"] is not None:
            P = lv["P"]
            out[f"L{l}_P_crow"] = P.crow_indices().numpy().astype(np.int32)
            out[f"L{l}_P_col"] = P.col_indices().numpy().astype(np.int32)
            out[f"L{l}_P_val"] = P.values().numpy()
            out[f"L{l}_P_shape"] = np.array(P.shape)
    with contextlib.redirect_stdout(io.StringIO()):
        bs = amg.Dhalf_inv * b if amg.Dhalf_inv is not None else b
        out["vcycle1"] = amg._v_cycle(0, torch.zeros_like(bs), bs).numpy()
        out["solve_x"] = amg.solve(b, tol=1e-30, max_iter=4).numpy()
        out["apply_x"] = amg.apply(b, cycles=2).numpy()
        # update with the next step's values (frozen hierarchy, new Galerkin products)
        A2 = torch.sparse_csr_tensor(torch.from_numpy(crow), torch.from_numpy(col),
                                     torch.from_numpy(traj["A_val_all"][1]), size=A.shape)
        amg.update_matrix(A2)
        for l, lv in enumerate(amg.levels):
            out[f"U{l}_A_val"] = lv["A"].values().numpy()
            out[f"U{l}_A_crow"] = lv["A"].crow_indices().numpy().astype(np.int32)
            out[f"U{l}_A_col"] = lv["A"].col_indices().numpy().astype(np.int32)
            out[f"U{l}_inv_relax"] = lv["inv_relax"].numpy()
        b2 = torch.from_numpy(traj["b_all"][1])
        out["update_solve_x"] = amg.solve(b2, tol=1e-30, max_iter=3).numpy()
    out["b"] = traj["b0"]
    out["b2"] = traj["b_all"][1]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "levels", [lv["n"] for lv in amg.levels])


def main():
    # two-phase 2-D, config-0 physics on a 32x32 grid (small enough for a fixture)
    cfg, f = scenarios.two_phase_2d(seed=0, nx=32, ny=32, nz=1, steps=4)
    t0 = run_trajectory("two_phase_32x32", cfg, f, steps=4, dt_days=1.0)
    amg_fixture("amg_two_phase_32x32", t0)
    # the 64x64x1 configuration itself, first two steps
    cfg, f = scenarios.two_phase_2d(seed=0, steps=2)
    run_trajectory("two_phase_64x64", cfg, f, steps=2, dt_days=1.0)
    # the adjoint sub-case grid: 16x16x2, sigma 0.7, dt 2 d (gravity active)
    cfg, f = scenarios.adjoint_case(seed=3, nx=16, ny=16, nz=2, steps=10)
    run_trajectory("two_phase_16x16x2", cfg, f, steps=10, dt_days=2.0)
    # black oil 5-spot physics (PVT, Stone II, gravity, capillarity) on 10x10x4
    cfg, f = scenarios.black_oil_5spot(seed=1, nx=10, ny=10, nz=4, steps=5, inj_rate=20.0)
    run_trajectory("black_oil_10x10x4", cfg, f, steps=5, dt_days=5.0)
    # gas-injection physics (surface-rate gas injectors, BHP producers) on 12x12x3
    # (the 2e5 sm3/d stress rate makes the reference's own saturation update diverge
    # on small grids, so the trajectory fixture uses a rate its explicit update can carry)
    cfg, f = scenarios.gas_injection_1m(seed=2, nx=12, ny=12, nz=3, steps=4, gas_rate=1.0e2,
                                        n_inj_side=1, n_prod_side=2, surface_units=True,
                                        rate_scale=1.0)
    cfg["fluid"]["capillary_pressure_og"] = {"pc_scale": 2.0e4, "pc_exponent": 1.5}
    cfg["wells"].append({"name": "PS", "type": "producer", "i": 6, "j": 2, "k": 0, "radius": 0.1,
                         "control_type": "rate", "control_value": 5.0, "rate_type": "surface",
                         "surface_phase": "oil", "limits": {"wopr": 3.0}})
    run_trajectory("gas_injection_12x12x3", cfg, f, steps=4, dt_days=2.0)
    # the reference's default pressure solver (Jacobi-PCG): solves of a recorded
    # system, and a whole trajectory on a case where its absolute tolerance is met
    # (a rate producer; with a BHP producer the well row keeps sqrt(r.M^-1 r) large)
    pcg_fixture("pcg_two_phase_32x32", t0, [(1e-6, 25), (1e-6, 120)])
    cfg, f = scenarios.two_phase_2d(seed=5, nx=20, ny=16, nz=2, steps=3)
    cfg["wells"][1] = {"name": "PROD", "type": "producer", "i": 19, "j": 15, "k": 0, "radius": 0.1,
                       "control_type": "rate", "control_value": 40.0}
    cfg["simulation"]["cg_tolerance"] = 1e-9
    cfg["simulation"]["cg_max_iter"] = 3000
    run_trajectory("cg_two_phase_20x16x2", cfg, f, steps=3, dt_days=1.0, solver="cg")
    three_phase_fixture()
    well_fixtures()
    amg_3d_fixtures()


def three_phase_fixture():
    """Three phases without PVT (initial free gas above Sgc, a gas and a water
    injector, two rate producers): the reference's constant-compressibility gas
    path, which the black-oil fixtures do not reach.  Also its trajectory under
    the reference's own Jacobi-PCG (pressure_solver "cg")."""
    cfg, f = scenarios.three_phase(seed=6, steps=5)
    run_trajectory("three_phase_16x16x3", cfg, f, steps=5, dt_days=1.0)
    cfg, f = scenarios.three_phase(seed=6, steps=3)
    cfg["simulation"]["cg_tolerance"] = 1e-9
    cfg["simulation"]["cg_max_iter"] = 3000
    run_trajectory("cg_three_phase_16x16x3", cfg, f, steps=3, dt_days=1.0, solver="cg")


def _well_case(nx, ny, wells, s_w, s_g, rv_max=0.0, k_md=150.0, poro=0.22):
    """A small homogeneous black-oil grid (10 x 10 x 8 m cells, Stone II) around
    a handful of surface-rate wells."""
    pvt = scenarios.pvt_table_black_oil(rv_max=rv_max)
    shape = (nx, ny, 1)
    k = np.full(shape, k_md * scenarios.MD)
    cfg = {
        "reservoir": {"dimensions": [nx, ny, 1], "grid_size": [10.0, 10.0, 8.0], "porosity": poro,
                      "permeability": k_md, "k_vertical_fraction": 1.0, "c_rock": 1e-5},
        "fluid": {"pressure": 21.0, "s_w": s_w, "s_g": s_g, "pvt": {"table": pvt},
                  "rho_oil": 850.0, "rho_water": 1000.0, "rho_gas": 1.0,
                  "relative_permeability": {"model": "stone2", "nw": 2.0, "no": 2.0, "ng": 2.0,
                                            "sw_cr": 0.2, "so_r": 0.2, "sg_cr": 0.0}},
        "wells": wells,
        "simulation": {"solver_type": "impes", "time_step_days": 1.0, "total_time_days": 3.0},
    }
    return cfg, {"kx": k, "ky": k.copy(), "kz": k.copy(), "poro": np.full(shape, poro)}


def well_fixtures():
    """Surface-rate wells as the reference's own tests place them
    (tests/test_surface_*.py, tests/test_component_balance_rv.py): a surface oil
    producer beside a water injector, a surface gas producer in free gas, a
    surface gas injector with a surface liquid producer on a table with Rv, and
    a surface water injector beside a reservoir-rate producer; 3 steps of 1 day."""
    w = lambda name, typ, i, j, **kw: dict(name=name, type=typ, i=i, j=j, k=0, radius=0.1,
                                            control_type="rate", **kw)
    cases = {
        "wells_surface_oil_6x6": _well_case(6, 6, [
            w("PO", "producer", 4, 4, control_value=60.0, rate_type="surface", surface_phase="oil"),
            w("WI", "injector", 1, 1, control_value=50.0, injected_phase="water")], 0.3, 0.0),
        "wells_surface_gas_6x6": _well_case(6, 6, [
            w("PG", "producer", 3, 3, control_value=25.0, rate_type="surface", surface_phase="gas")],
            0.3, 0.06),
        "wells_rv_liquid_6x6": _well_case(6, 6, [
            w("GI", "injector", 1, 1, control_value=300.0, rate_type="surface", injected_phase="gas"),
            w("PL", "producer", 4, 4, control_value=150.0, rate_type="surface", surface_phase="liquid")],
            0.25, 0.05, rv_max=1.0e-4),
        "wells_surface_water_6x6": _well_case(6, 6, [
            w("WI", "injector", 2, 2, control_value=80.0, rate_type="surface", injected_phase="water"),
            w("PR", "producer", 4, 4, control_value=70.0)], 0.2, 0.0),
    }
    for name, (cfg, f) in cases.items():
        run_trajectory(name, cfg, f, steps=3, dt_days=1.0)


def amg_3d_fixtures():
    """ClassicalAMG hierarchies of 3-D pressure matrices: black-oil 10x10x4
    (PVT, gravity, capillarity, anisotropic kz) and the three-phase 16x16x3."""
    for name, traj, seed, coarsest in (("amg_black_oil_10x10x4", "black_oil_10x10x4", 7, 20),
                                       ("amg_three_phase_16x16x3", "three_phase_16x16x3", 11, 40)):
        amg_fixture(name, dict(np.load(os.path.join(HERE, f"{traj}.npz"))), seed=seed, coarsest=coarsest)


def config_fixtures(which=("config0", "config3", "config1")):
    """The benchmark configurations at their stated sizes: the 64x64x1
    oil-water case for all of its 100 daily steps, the 64x64x8 adjoint-case grid
    for its 50 two-day steps, and a two-step spot check of the 100x100x20
    black-oil 5-spot (200,000 cells, about 150 s per direct solve).  Whole
    fields are kept at a few steps and 2,048 fixed cells at every step."""
    runs = {
        "config0": ("config0_64x64x1_100steps", "two_phase_2d", {"seed": 0, "steps": 100}, 100, 1.0,
                    {1, 10, 25, 50, 75, 100}),
        "config3": ("config3_64x64x8_50steps", "adjoint_case", {"seed": 3, "steps": 50}, 50, 2.0,
                    {1, 25, 50}),
        "config1": ("config1_100x100x20_2steps", "black_oil_5spot", {"seed": 1, "steps": 2}, 2, 5.0, {2}),
    }
    for key in which:
        name, fn, kwargs, steps, dt_days, full_at = runs[key]
        cfg, f = getattr(scenarios, fn)(**kwargs)
        run_trajectory(name, cfg, f, steps=steps, dt_days=dt_days, full_at=full_at, n_samples=2048,
                       keep_systems=1, generator=(fn, kwargs))


def reference_producer_rates(cfg, fields, steps, dt, grad=False):
    """Producer oil rates [steps x producers] (m3/day) of the reference's own IMPES
    steps with the pressure solved densely (torch.linalg.solve, so autograd runs
    through it), and -- with grad -- the leaf tensors (delta ln k of every cell,
    scaling kx, ky and kz together, and porosity) to differentiate against.

    The rate is the flux balance of the producer's pressure row built from the
    reference's own terms: q = sum_f c_f (p_nb - p_c) - acc_c (p_c - p_prev,c)
    + Qg_c, times the oil fractional flow mob_o / (mob_t + 1e-10) at the step's
    starting state.  c_f are the upwinded face coefficients the reference hands
    to _build_pressure_matrix_vectorized, acc = PV ct / dt as that function forms
    it, and Qg the gravity part of _build_pressure_rhs (its right-hand side with
    the well terms zeroed, less the accumulation term).  The well's own
    WI lambda (p_c - p_bhp) is the same number algebraically but round-off."""
    shape = fields["kx"].shape
    delta = torch.zeros(shape, dtype=torch.float64, requires_grad=grad)
    poro = torch.tensor(np.array(fields["poro"]), dtype=torch.float64).requires_grad_(grad)
    rec = {}
    orig_mat, orig_rhs = Simulator._build_pressure_matrix_vectorized, Simulator._build_pressure_rhs

    def mat(self, Tx, Ty, Tz, dt_, wb):
        try:
            ct = self.fluid.calc_total_compressibility(self.fluid.pressure, self.fluid.s_w, self.fluid.s_g)
            acc = self.porous_volume.view(-1) * ct.view(-1) / dt_
        except Exception:
            acc = self.porous_volume.view(-1) * self.fluid.cf.view(-1) / dt_
        rec.update(T=(Tx, Ty, Tz), acc=acc)
        return orig_mat(self, Tx, Ty, Tz, dt_, wb)

    def rhs(self, dt_, P_prev, mob_w, mob_o, mob_g, q_wells, dpx, dpy, dpz):
        Q = orig_rhs(self, dt_, P_prev, mob_w, mob_o, mob_g, q_wells, dpx, dpy, dpz)
        Q0 = orig_rhs(self, dt_, P_prev, mob_w, mob_o, mob_g, torch.zeros_like(q_wells), dpx, dpy, dpz)
        rec.update(Qg=Q0 - rec["acc"] * P_prev.reshape(-1), P_prev=P_prev, mob=(mob_w, mob_o, mob_g))
        return Q

    def dense(A, b, **kw):
        x = torch.linalg.solve(A.to_dense(), b)
        rec["p_new"] = x
        return x

    Simulator._build_pressure_matrix_vectorized = mat
    Simulator._build_pressure_rhs = rhs
    pamg.amg_solve = dense
    try:
        f = dict(fields)
        scale = torch.exp(delta)
        f["kx"] = torch.tensor(np.array(fields["kx"])) * scale
        f["ky"] = torch.tensor(np.array(fields["ky"])) * scale
        f["kz"] = torch.tensor(np.array(fields["kz"])) * scale
        with tempfile.TemporaryDirectory() as td:
            with contextlib.redirect_stdout(io.StringIO()):
                res = Reservoir(cfg["reservoir"], torch.device("cpu"))
                res.permeability_x, res.permeability_y, res.permeability_z = f["kx"], f["ky"], f["kz"]
                res.porosity = poro
                res.porous_volume = res.cell_volume * poro
                wm = WellManager(cfg["wells"], res)
                fl = Fluid(cfg["fluid"], res, torch.device("cpu"))
                sim_cfg = dict(cfg["simulation"], pressure_solver="amg")
                sim = Simulator(res, fl, wm, sim_cfg, torch.device("cpu"))
            prods = [w for w in wm.get_wells() if w.type == "producer"]
            nx, ny, nz = shape
            out = []
            for _ in range(steps):
                with contextlib.redirect_stdout(io.StringIO()):
                    assert sim.run_step(dt)
                Tx, Ty, Tz = rec["T"]
                P = rec["p_new"].reshape(shape)
                Pp = rec["P_prev"].reshape(-1)
                Fx = Tx * (P[:-1] - P[1:])
                Fy = Ty * (P[:, :-1] - P[:, 1:])
                Fz = Tz * (P[:, :, :-1] - P[:, :, 1:])
                z = torch.zeros
                inflow = (torch.cat([z(1, ny, nz), Fx], 0) - torch.cat([Fx, z(1, ny, nz)], 0)
                          + torch.cat([z(nx, 1, nz), Fy], 1) - torch.cat([Fy, z(nx, 1, nz)], 1)
                          + torch.cat([z(nx, ny, 1), Fz], 2) - torch.cat([Fz, z(nx, ny, 1)], 2)).reshape(-1)
                mw, mo, mg = (m.reshape(-1) for m in rec["mob"])
                pn = P.reshape(-1)
                row = []
                for w in prods:
                    c = (w.i * ny + w.j) * nz + w.k
                    qfb = inflow[c] - rec["acc"][c] * (pn[c] - Pp[c]) + rec["Qg"][c]
                    row.append(qfb * (mo[c] / (mw[c] + mo[c] + mg[c] + 1e-10)) * 86400.0)
                out.append(torch.stack(row))
    finally:
        Simulator._build_pressure_matrix_vectorized = orig_mat
        Simulator._build_pressure_rhs = orig_rhs
    return torch.stack(out), delta, poro


def adjoint_fixture(steps=6):
    """Autograd through the reference's own IMPES step with a dense pressure
    solve on the 16x16x2 sub-case of the adjoint workload: the misfit J of the
    flux-balance producer oil rates against the rates of the seed-5 permeability
    field, and dJ/d ln k, dJ/d porosity."""
    cfg, f = scenarios.adjoint_case(seed=3, steps=steps, nx=16, ny=16, nz=2)
    _, f2 = scenarios.adjoint_case(seed=5, steps=steps, nx=16, ny=16, nz=2)
    dt = cfg["simulation"]["time_step_days"] * 86400.0
    with torch.no_grad():
        target, _, _ = reference_producer_rates(cfg, dict(f2, poro=f["poro"]), steps, dt)
    q, delta, poro = reference_producer_rates(cfg, f, steps, dt, grad=True)
    J = ((q - target) ** 2).sum()
    g_lnk, g_poro = torch.autograd.grad(J, (delta, poro))
    out = dict(cfg=json.dumps(cfg), kx=f["kx"], ky=f["ky"], kz=f["kz"], poro=f["poro"], dt=dt, steps=steps,
               target=target.numpy(), rates=q.detach().numpy(), J=float(J.detach()),
               g_lnk=g_lnk.numpy().reshape(-1), g_poro=g_poro.numpy().reshape(-1))
    np.savez_compressed(os.path.join(HERE, "adjoint_ref_16x16x2.npz"), **out)
    print("adjoint_ref_16x16x2 J", out["J"], "|g_lnk|", np.linalg.norm(out["g_lnk"]),
          "|g_poro|", np.linalg.norm(out["g_poro"]), flush=True)


def main_pcg_only():
    """Regenerate only the Jacobi-PCG fixtures (the others are unchanged)."""
    cfg, f = scenarios.two_phase_2d(seed=0, nx=32, ny=32, nz=1, steps=4)
    t0 = dict(np.load(os.path.join(HERE, "two_phase_32x32.npz")))
    pcg_fixture("pcg_two_phase_32x32", t0, [(1e-6, 25), (1e-6, 120)])
    cfg, f = scenarios.two_phase_2d(seed=5, nx=20, ny=16, nz=2, steps=3)
    cfg["wells"][1] = {"name": "PROD", "type": "producer", "i": 19, "j": 15, "k": 0, "radius": 0.1,
                       "control_type": "rate", "control_value": 40.0}
    cfg["simulation"]["cg_tolerance"] = 1e-9
    cfg["simulation"]["cg_max_iter"] = 3000
    run_trajectory("cg_two_phase_20x16x2", cfg, f, steps=3, dt_days=1.0, solver="cg")


if __name__ == "__main__":
    if "--pcg-only" in sys.argv:
        main_pcg_only()
        sys.exit(0)
    if "--three-phase-only" in sys.argv:
        three_phase_fixture()
        sys.exit(0)
    if "--wells-only" in sys.argv:
        well_fixtures()
        sys.exit(0)
    if "--amg-3d-only" in sys.argv:
        amg_3d_fixtures()
        sys.exit(0)
    if "--adjoint-only" in sys.argv:
        adjoint_fixture()
        sys.exit(0)
    if "--configs-only" in sys.argv:
        sel = [a.split("=", 1)[1] for a in sys.argv if a.startswith("--which=")]
        config_fixtures(tuple(sel[0].split(",")) if sel else ("config0", "config3", "config1"))
        sys.exit(0)
    main()
