"""Full IMPES steps on the GPU against the reference trajectories (direct-solve
pressure oracle) and the drop-in API."""
import json
import os

import numpy as np
import pytest
import torch

from gpu_util import cfg_fields, gpu_sim, oracle_model, to_np

pytestmark = pytest.mark.gpu

CASES = ["two_phase_32x32", "two_phase_64x64", "two_phase_16x16x2", "black_oil_10x10x4",
         "gas_injection_12x12x3", "three_phase_16x16x3", "wells_surface_oil_6x6",
         "wells_surface_gas_6x6", "wells_rv_liquid_6x6", "wells_surface_water_6x6"]


def solve_tol(cfg):
    """FGMRES tolerance (Jacobi-scaled relative residual) for a parity run.

    With a BHP well the well row anchors the pressure level and 1e-13 is well
    above the residual's rounding floor.  With rate wells only, nothing but the
    accumulation term PV*c_t/dt anchors it, so ||D^-1 b|| is small against ||x||:
    the exact solution's own relative residual is ~3.5e-13 on the three-phase
    16x16x3 system, with a rounding floor near 8.5e-13.  A 1e-13 request there
    can never be met (every step would be retried at dt/2), so those cases ask
    for 1e-11, which bounds the pressure error near 6e-10 relative."""
    bhp = any(str(w.get("control_type", w.get("control", {}).get("type", ""))) == "bhp"
              for w in cfg["wells"])
    return 1e-13 if bhp else 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", CASES)
def test_trajectory_matches_reference(golden, name, precision):
    """p to 1e-8 relative and Sw/Sg to 1e-8 absolute at every step against the
    reference's trajectory with an exact pressure solve."""
    g = golden(name)
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=solve_tol(cfg), norm="jacobi", precision=precision,
                            max_iters=400, restart=40)
    dt = float(g["dt"])
    for s in range(g["p"].shape[0]):
        assert sim.run_step(dt)
        assert sim.last_krylov["converged"], (s, sim.last_krylov)
        p = to_np(fl.pressure)
        assert np.abs(p - g["p"][s]).max() <= 1e-8 * np.abs(g["p"][s]).max(), (s, sim.last_krylov)
        assert np.abs(to_np(fl.s_w) - g["sw"][s]).max() <= 1e-8
        assert np.abs(to_np(fl.s_g) - g["sg"][s]).max() <= 1e-8
    mb = sim.mass_balance
    got = np.array([mb[ph][io] for ph in ("water", "oil", "gas") for io in ("in", "out")])
    ref = g["balances"][-1][:6]
    assert np.all(np.abs(got - ref) <= 1e-6 * np.maximum(np.abs(ref), 1e-9))


def test_reference_vcycle_mode_matches_oracle(golden):
    """pressure_solver='amg': stand-alone V-cycles with the reference's stopping
    rule, compared with the oracle's restatement of amg_solve (same tie-break)."""
    from oracle.amg import AMGSolver
    g = golden("two_phase_32x32")
    cfg, f = cfg_fields(g)
    cfg["simulation"]["pressure_solver"] = "amg"
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-30, max_cycles=6, coarsest_size=50, seed=4)
    m = oracle_model(g)
    solver = AMGSolver(tol=1e-30, max_cycles=6, coarsest_size=50, seed=4)
    dt = float(g["dt"])
    for _ in range(2):
        sim.run_step(dt)
        m.step(dt, solve=solver)
        p = to_np(fl.pressure)
        assert np.abs(p - m.p).max() <= 1e-7 * np.abs(m.p).max()
        assert np.abs(to_np(fl.s_w) - m.sw).max() <= 1e-7


def test_mixed_precision_drift_small(golden):
    """fp32 V-cycle inside fp64 FGMRES: saturation drift vs the fp64 path < 1e-6."""
    g = golden("black_oil_10x10x4")
    cfg, f = cfg_fields(g)
    _, f64, _, s64 = gpu_sim(cfg, f, tol=1e-10, precision="fp64")
    _, f32, _, s32 = gpu_sim(cfg, f, tol=1e-10, precision="mixed")
    for _ in range(5):
        s64.run_step(float(g["dt"]))
        s32.run_step(float(g["dt"]))
    assert np.abs(to_np(f64.s_w) - to_np(f32.s_w)).max() < 1e-6
    assert np.abs(to_np(f64.pressure) - to_np(f32.pressure)).max() < 1e-6 * to_np(f64.pressure).max()


def test_step_is_deterministic(golden):
    g = golden("two_phase_16x16x2")
    cfg, f = cfg_fields(g)
    outs = []
    for _ in range(2):
        _, fl, _, sim = gpu_sim(cfg, f, tol=1e-10)
        for _ in range(3):
            sim.run_step(float(g["dt"]))
        outs.append((fl.pressure.clone(), fl.s_w.clone()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


def test_dropin_modules_and_json_schema(tmp_path):
    """The reference's import paths and both well schemas; PVT from a JSON file."""
    from impes_b200 import scenarios
    from simulator.fluid import Fluid
    from simulator.reservoir import Reservoir
    from simulator.simulation import Simulator
    from simulator.well import WellManager
    from solver.pressure_amg import amg_solve
    from solver.classical_amg import ClassicalAMG  # noqa: F401
    pvt_path = tmp_path / "pvt.json"
    pvt_path.write_text(json.dumps(scenarios.pvt_table_black_oil()))
    cfg = {
        "reservoir": {"dimensions": [8, 6, 3], "grid_size": [10.0, 10.0, 4.0], "porosity": 0.22,
                      "permeability": 120.0, "k_vertical_fraction": 0.2},
        "fluid": {"pressure": 22.0, "s_w": 0.25, "s_g": 0.02, "pvt_path": str(pvt_path),
                  "relative_permeability": {"model": "stone2", "nw": 2, "ng": 2.5}},
        "wells": [
            {"name": "I", "type": "injector", "coordinates": [0, 0, 1], "radius": 0.1,
             "control": {"type": "rate", "value": 20.0}, "injected_phase": "water"},
            # a rate producer: a BHP producer's saturation-step rate WI*lambda*(p - p_bhp)
            # is the rounding of p when the cell sits at p_bhp (simulation.py:1297)
            {"name": "P", "type": "producer", "i": 7, "j": 5, "k": 1, "radius": 0.1,
             "control_type": "rate", "control_value": 15.0},
        ],
        "simulation": {"solver_type": "impes", "pressure_solver": "gmres_amg",
                       "amg": {"tol": 1e-12, "max_iters": 300}},
    }
    dev = torch.device("cuda")
    res = Reservoir(cfg["reservoir"], dev)
    wm = WellManager(cfg["wells"], res)
    fl = Fluid(cfg["fluid"], res, dev)
    sim = Simulator(res, fl, wm, cfg["simulation"], dev)
    assert sim.run_step(86400.0)
    from oracle.impes import Model
    m = Model(cfg)
    m.step(86400.0)
    assert np.abs(to_np(fl.pressure) - m.p).max() <= 1e-8 * np.abs(m.p).max()
    assert np.abs(to_np(fl.s_w) - m.sw).max() <= 1e-8
    assert np.abs(to_np(fl.s_g) - m.sg).max() <= 1e-8
    assert wm.get_wells()[1].cell_index_flat == (7 * 6 + 5) * 3 + 1
    # amg_solve keeps the reference's signature and returns b's dtype
    rowptr, col, val, rhs = sim.assemble(86400.0)
    A = torch.sparse_csr_tensor(rowptr.long(), col.long(), val, size=(rhs.numel(),) * 2)
    x = amg_solve(A, rhs.float(), tol=1e-6, max_cycles=5)
    assert x.dtype == torch.float32 and x.shape == rhs.shape


def test_bhp_min_autoswitch_and_limits():
    """bhp_min never reduces the outflow (the reference's assertion,
    tests/test_phase_limits_and_autoswitch.py:70-71).  With the reference's sign
    convention the producer's required BHP is p_block + |q|/(WI lambda), never
    below bhp_min, so the switch at simulation.py:1636-1650 does not fire; a
    surface oil limit throttles the rate."""
    from impes_b200 import scenarios
    from impes_b200.simulator import build_from_config
    base = {
        "reservoir": {"dimensions": [5, 5, 1], "grid_size": [10, 10, 10], "porosity": 0.2,
                      "permeability": 100.0, "k_vertical_fraction": 1.0},
        "fluid": {"pressure": 10.0, "s_w": 0.2, "s_g": 0.0, "pvt": {"table": scenarios.pvt_table_black_oil()}},
        "simulation": {"solver_type": "impes", "pressure_solver": "gmres_amg",
                       "amg": {"tol": 1e-12, "coarsest_size": 10}},
    }
    cfg1 = json.loads(json.dumps(base))
    cfg1["wells"] = [{"name": "P1", "type": "producer", "i": 2, "j": 2, "k": 0, "radius": 0.1,
                      "control_type": "rate", "control_value": 20000.0}]
    cfg2 = json.loads(json.dumps(base))
    cfg2["wells"] = [{"name": "P2", "type": "producer", "i": 2, "j": 2, "k": 0, "radius": 0.1,
                      "control_type": "rate", "control_value": 20000.0, "bhp_min": 9.5}]
    _, _, wm1, s1 = build_from_config(cfg1, device="cuda")
    _, _, wm2, s2 = build_from_config(cfg2, device="cuda")
    s1.run_step(86400.0)
    s2.run_step(86400.0)
    q1 = abs(wm1.get_wells()[0].last_q_total or 0.0)
    q2 = abs(wm2.get_wells()[0].last_q_total or 0.0)
    assert q2 <= q1 + 1e-9
    assert wm1.get_wells()[0].last_mode == "rate" and wm2.get_wells()[0].last_mode == "rate"
    cfg3 = json.loads(json.dumps(base))
    cfg3["fluid"].update({"pressure": 20.0, "s_w": 0.3, "s_g": 0.02})
    cfg3["wells"] = [{"name": "PS", "type": "producer", "i": 2, "j": 2, "k": 0, "radius": 0.1,
                      "control_type": "rate", "control_value": 50000.0, "rate_type": "surface",
                      "surface_phase": "oil", "limits": {"wopr": 100.0}}]
    _, _, wm3, s3 = build_from_config(cfg3, device="cuda")
    s3.run_step(86400.0)
    assert wm3.get_wells()[0].last_surface_rates["oil"] <= 100.0 * 1.10


@pytest.mark.parametrize("name", ["cg_two_phase_20x16x2", "cg_three_phase_16x16x3"])
def test_reference_cg_solver_matches_reference(golden, name):
    """pressure_solver "cg": the reference's own Jacobi-PCG path end to end
    (simulation.py:931-966, 1662-1697), against the trajectory the reference
    produced with it (two phases, and three phases with free gas)."""
    g = golden(name)
    cfg, f = cfg_fields(g)
    assert cfg["simulation"]["pressure_solver"] == "cg"
    _, fl, _, sim = gpu_sim(cfg, f)
    for s in range(g["p"].shape[0]):
        assert sim.run_step(float(g["dt"]))
        assert sim.last_krylov["converged"]
        assert np.abs(to_np(fl.pressure) - g["p"][s]).max() <= 1e-9 * np.abs(g["p"][s]).max()
        assert np.abs(to_np(fl.s_w) - g["sw"][s]).max() <= 1e-9


def test_pcg_entry_point_matches_reference_iterates(golden):
    """impes_pcg_solve after a fixed number of iterations equals the reference's
    _solve_pressure_cg_pytorch iterate (a BHP system: the absolute tolerance is
    not met, so both stop at max_iter)."""
    import ctypes as C
    from impes_b200 import _lib
    g = golden("pcg_two_phase_32x32")
    n = len(g["A0_crow"]) - 1
    dev = torch.device("cuda")
    rowptr = torch.tensor(g["A0_crow"], dtype=torch.int32, device=dev)
    col = torch.tensor(g["A0_col"], dtype=torch.int32, device=dev)
    val = torch.tensor(g["A0_val"], device=dev)
    b = torch.tensor(g["b0"], device=dev)
    for q, (tol, it) in enumerate(zip(g["tol"], g["max_iter"])):
        x = torch.full((n,), 3.0, dtype=torch.float64, device=dev)
        iters, conv, rz = C.c_int(), C.c_int(), C.c_double()
        st = _lib.lib.impes_pcg_solve(n, _lib.ptr(rowptr), _lib.ptr(col), _lib.ptr(val), _lib.ptr(b),
                                      _lib.ptr(x), float(tol), int(it), C.byref(iters), C.byref(conv),
                                      C.byref(rz), _lib.stream_of(dev))
        assert st == 0 and iters.value == int(it) and bool(conv.value) == bool(g[f"converged{q}"])
        ref = g[f"x{q}"]
        assert np.abs(to_np(x) - ref).max() <= 1e-9 * np.abs(ref).max()


def test_run_writes_reference_result_files(tmp_path):
    """Simulator.run: the reference's results directory, txt summary and npz keys
    (simulation.py:2121-2248), intermediate states at its save_interval cadence."""
    import glob
    import os
    from impes_b200 import scenarios
    from impes_b200.simulator import build_from_config
    cfg, f = scenarios.two_phase_2d(seed=2, nx=10, ny=8, nz=1, steps=4)
    cfg["simulation"].update({"total_time_days": 4.0, "time_step_days": 1.0, "save_interval": 2})
    _, fl, _, sim = build_from_config(cfg, f, device="cuda")
    out = sim.run("case", results_root=str(tmp_path))
    assert os.path.basename(out).startswith("case_")
    snaps = sorted(glob.glob(os.path.join(out, "intermediate", "case_step_*.npz")))
    assert [os.path.basename(s) for s in snaps] == ["case_step_2.npz", "case_step_4.npz"]
    z = np.load(os.path.join(out, "case.npz"))
    assert sorted(z.files) == ["pressure", "sg", "so", "sw"]
    assert np.array_equal(z["pressure"], fl.pressure.cpu().numpy())
    txt = open(os.path.join(out, "case.txt")).read()
    assert txt.startswith("=== SUMMARY (final) ===\nPressure MPa: min=")
    assert "=== MASS BALANCE (kg) ===" in txt and "total net=" in txt
    assert sim.step_count == 4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_whole_step_graph_matches_host_driven_steps(golden, monkeypatch, precision):
    """From the second step on, an FGMRES step runs as one CUDA graph (assembly,
    Galerkin update, device-driven FGMRES under a conditional WHILE node,
    saturation).  Its trajectory equals the host-driven step's to rounding
    (the device solver sums its norms in another order) and the reference's
    at 1e-8."""
    g = golden("gas_injection_12x12x3")
    cfg, f = cfg_fields(g)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("IMPES_NO_STEP_GRAPH", flag)
        _, fl, _, sim = gpu_sim(cfg, f, tol=1e-13, norm="jacobi", precision=precision, max_iters=400,
                                restart=40)
        traj = []
        for s in range(g["p"].shape[0]):
            assert sim.run_step(float(g["dt"]))
            assert sim.last_krylov["converged"], sim.last_krylov
            traj.append((to_np(fl.pressure), to_np(fl.s_w), to_np(fl.s_g), sim.last_krylov["iterations"]))
            assert np.abs(traj[-1][0] - g["p"][s]).max() <= 1e-8 * np.abs(g["p"][s]).max()
            assert np.abs(traj[-1][1] - g["sw"][s]).max() <= 1e-8
        out[flag] = traj
        graphs, refused = sim.step_graphs()
        assert not refused and (graphs >= 1) == (flag == "0"), (flag, graphs, refused)
        sim.close()
    # At tol 1e-13 the solve ends a few digits above its rounding floor: the two
    # paths sum their dots in different orders, and the fp32 V-cycle turns that
    # into a slightly different Krylov tail (a step or two), never a systematic
    # excess.
    step_slack = 1 if precision == "fp64" else 3
    for (p1, w1, s1, i1), (p0, w0, s0, i0) in zip(out["1"], out["0"]):
        assert np.abs(p1 - p0).max() <= 1e-11 * np.abs(p1).max()
        assert np.abs(w1 - w0).max() <= 1e-11 and np.abs(s1 - s0).max() <= 1e-11
        assert abs(i1 - i0) <= step_slack, (i1, i0)
    tot1, tot0 = sum(t[3] for t in out["1"]), sum(t[3] for t in out["0"])
    assert abs(tot1 - tot0) <= 0.05 * tot1 + 2, (tot1, tot0)


def test_whole_step_graph_failed_solve_leaves_state(golden):
    """A step graph whose solve misses its tolerance restores the pressure and
    skips the saturation update on the device; run_step retries at dt/2 as the
    reference does and reports failure, with the state untouched."""
    g = golden("two_phase_16x16x2")
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-10, norm="jacobi", max_iters=400, restart=40)
    assert sim.run_step(float(g["dt"]))             # builds the hierarchy (host path)
    assert sim.run_step(float(g["dt"]))             # first step graph
    p0, w0 = fl.pressure.clone(), fl.s_w.clone()
    sim.amg_max_iters = 1
    sim.amg_tol = 1e-30
    sim.sim_params["max_time_step_attempts"] = 2
    assert not sim.run_step(float(g["dt"]))
    assert torch.equal(fl.pressure, p0) and torch.equal(fl.s_w, w0)
    sim.amg_max_iters, sim.amg_tol = 400, 1e-10
    assert sim.run_step(float(g["dt"]))


@pytest.mark.parametrize("graph", ["1", "0"])
def test_quadratic_warm_start_matches_reference(golden, monkeypatch, graph):
    """warm_start "quadratic": FGMRES starts from the parabola through the last
    three accepted pressures (linear while only two exist).  Only the first
    iterate changes, so the trajectory still equals the reference's at 1e-8,
    on the whole-step graph and on the host-driven step."""
    monkeypatch.setenv("IMPES_NO_STEP_GRAPH", graph)
    g = golden("config0_64x64x1_100steps")
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-13, norm="jacobi", precision="mixed", max_iters=1000, restart=60,
                            warm_start="quadratic")
    idx = g["sample_idx"]
    dt = float(g["dt"])
    for st in range(1, 21):
        assert sim.run_step(dt), st
        assert sim.last_krylov["converged"], (st, sim.last_krylov)
        p, sw = to_np(fl.pressure), to_np(fl.s_w)
        ps = g["p_s"][st - 1]
        assert np.abs(p[idx] - ps).max() <= 1e-8 * np.abs(ps).max(), st
        assert np.abs(sw[idx] - g["sw_s"][st - 1]).max() <= 1e-8, st
    graphs, refused = sim.step_graphs()
    assert not refused and (graphs >= 1) == (graph == "0"), (graphs, refused)
    sim.close()
