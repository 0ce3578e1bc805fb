"""The benchmark's workloads as defined in impes_b200.scenarios: sizes, wells,
solver settings and field statistics, so that a change to a generator cannot
silently change what bench.py measures."""
import math

import numpy as np

from impes_b200 import scenarios


def _wells(cfg, kind):
    return [w for w in cfg["wells"] if w["type"] == kind]


def test_million_cell_gas_injection_workload():
    cfg, f = scenarios.gas_injection_1m()
    assert cfg["reservoir"]["dimensions"] == [200, 200, 25]
    assert len(_wells(cfg, "injector")) == 9 and len(_wells(cfg, "producer")) == 16
    assert all(w["injected_phase"] == "gas" for w in _wells(cfg, "injector"))
    assert all(w["control_type"] == "bhp" and w["control_value"] == 15.0 for w in _wells(cfg, "producer"))
    sim = cfg["simulation"]
    assert sim["global_rate_scale"] == 0.05 and sim["max_substeps"] == 20
    assert sim["time_step_days"] == 2.0
    assert {k: sim["amg"][k] for k in ("tol", "theta", "max_levels", "coarsest_size")} == \
        {"tol": 1e-6, "theta": 0.2, "max_levels": 20, "coarsest_size": 120}
    assert f["kx"].shape == (200, 200, 25) and f["kx"].dtype == np.float64
    lnk = np.log(f["kx"] / scenarios.MD)
    assert abs(lnk.mean() - math.log(150.0)) < 0.05 and abs(lnk.std() - 1.0) < 0.05
    np.testing.assert_array_equal(f["kz"], 0.1 * f["kx"])
    assert 0.15 <= f["poro"].min() and f["poro"].max() <= 0.25
    cfg2, f2 = scenarios.gas_injection_1m()
    np.testing.assert_array_equal(f["kx"], f2["kx"])              # seeded


def test_ensemble_workload():
    cases = scenarios.ensemble(seed=4, members=64, steps=30)
    assert len(cases) == 64
    dims = [c[0]["reservoir"]["dimensions"] for c in cases]
    assert sum(int(np.prod(d)) for d in dims) == 3_089_408
    assert all(d[0] in (32, 48, 64, 96, 128) and d[1] in (32, 48, 64, 96, 128) and d[2] in (4, 8, 16)
               for d in dims)
    assert all(c[0]["simulation"]["time_step_days"] == 1.0 for c in cases)


def test_adjoint_and_small_workloads():
    cfg, f = scenarios.adjoint_case()
    assert cfg["reservoir"]["dimensions"] == [64, 64, 8] and cfg["simulation"]["time_step_days"] == 2.0
    assert len(cfg["wells"]) == 2 and cfg["fluid"]["s_g"] == 0.0
    cfg, _ = scenarios.black_oil_5spot()
    assert cfg["reservoir"]["dimensions"] == [100, 100, 20]
    assert len(_wells(cfg, "injector")) == 4 and len(_wells(cfg, "producer")) == 1
    cfg, _ = scenarios.two_phase_2d()
    assert cfg["reservoir"]["dimensions"] == [64, 64, 1] and len(cfg["wells"]) == 2
