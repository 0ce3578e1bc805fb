"""The concurrent ensemble driver against members stepped one at a time."""
import pytest
import torch

from impes_b200 import scenarios

pytestmark = pytest.mark.gpu


def _cases():
    dims = [(24, 16, 4), (8, 8, 2), (32, 24, 2), (12, 12, 4), (16, 8, 8), (20, 20, 1)]
    return [scenarios.two_phase_2d(seed=10 + q, nx=nx, ny=ny, nz=nz, steps=4, sigma=0.6)
            for q, (nx, ny, nz) in enumerate(dims)]


def test_ensemble_equals_single_runs():
    from impes_b200.ensemble import Ensemble
    from impes_b200.simulator import build_from_config
    cases = _cases()
    amg = {"tol": 1e-8, "norm": "jacobi"}
    ens = Ensemble(cases, workers=3, amg=amg)
    dt = 86400.0
    stats = ens.run(4, dt)
    assert all(s["status"] == 0 and s["steps"] == 4 for s in stats)
    assert len({s["worker"] for s in stats}) == 3
    for m, (cfg, f) in enumerate(cases):
        cfg = dict(cfg, simulation=dict(cfg["simulation"], amg=dict(cfg["simulation"]["amg"], **amg)))
        _, fl, _, sim = build_from_config(cfg, f, device="cuda")
        for _ in range(4):
            assert sim.run_step(dt)
        e = ens.sims[ens.members.index(m)].fluid
        assert torch.equal(e.pressure, fl.pressure), m
        assert torch.equal(e.s_w, fl.s_w), m
        sim.close()
    summ = ens.summary()
    assert [s["member"] for s in summ] == list(range(len(cases)))
    ens.close()


def test_ensemble_reports_member_failures():
    from impes_b200 import _lib
    from impes_b200.ensemble import Ensemble
    cases = _cases()[:3]
    ens = Ensemble(cases, workers=2, amg={"tol": 1e-30, "max_iters": 2, "norm": "jacobi"})
    with pytest.raises(_lib.NotConverged, match="member"):
        ens.run(2, 86400.0)
    assert all(s["status"] == _lib.ERR_NOT_CONVERGED and s["steps"] == 0 for s in ens.last_stats)
    ens.close()


def test_sharded_members_cover_the_ensemble():
    """Two ranks' shares, run one after the other on this GPU, give the same
    summaries as the whole ensemble on one rank."""
    from impes_b200.ensemble import Ensemble
    cases = _cases()
    whole = Ensemble(cases, workers=4)
    whole.run(2, 86400.0)
    ref = whole.summary()
    whole.close()
    parts = []
    for r in range(2):
        e = Ensemble(cases, rank=r, world=2, workers=2)
        e.run(2, 86400.0)
        parts += e.summary()
        e.close()
    parts.sort(key=lambda s: s["member"])
    assert [(s["member"], s["p_mean_MPa"], s["sw_mean"]) for s in parts] == \
        [(s["member"], s["p_mean_MPa"], s["sw_mean"]) for s in ref]
