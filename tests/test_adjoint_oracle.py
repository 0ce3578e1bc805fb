"""The adjoint checker (oracle/adjoint.py) against the pinned IMPES oracle and
against central finite differences of its own forward run."""
import numpy as np
import pytest
import torch

from impes_b200 import scenarios
from oracle import adjoint as oadj
from oracle.impes import Model


def _case(nx=16, ny=16, nz=2, seed=3, steps=3):
    cfg, f = scenarios.adjoint_case(seed=seed, nx=nx, ny=ny, nz=nz, steps=steps)
    dt = cfg["simulation"]["time_step_days"] * 86400.0

    def model(fields=f):
        return Model(cfg, fields["kx"], fields["ky"], fields["kz"], fields["poro"])
    return cfg, f, dt, model


def test_torch_forward_matches_oracle_step():
    _, _, dt, model = _case(nx=8, ny=8, nz=3)
    m = model()
    t = oadj.TorchIMPES(model())
    p, sw = torch.tensor(m.p), torch.tensor(m.sw)
    for _ in range(4):
        p, sw, rates = t.step(p, sw, t.lnk0, t.poro0, dt)
        m.step(dt)
        assert float((p - torch.tensor(m.p)).abs().max()) <= 1e-12 * float(np.abs(m.p).max())
        assert float((sw - torch.tensor(m.sw)).abs().max()) <= 1e-12
        assert len(rates) == 1 and np.isfinite(float(rates[0]))


def test_flux_balance_rate_equals_well_rate_when_well_term_resolves():
    """q_fb = WI*lambda_t*(p_c - p_bhp) algebraically: check it on a producer whose
    well term is not round-off (a tiny well index)."""
    cfg, f, dt, _ = _case(nx=6, ny=5, nz=2)
    m = Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"])
    prod = [w for w in m.wells if w.type == "producer"][0]
    prod.well_index = 1e-9
    t = oadj.TorchIMPES(m)
    p0, sw0 = torch.tensor(m.p), torch.tensor(m.sw)
    p1, _, rates = t.step(p0, sw0, t.lnk0, t.poro0, dt)
    c = m.cell(prod)
    mw, mo = t._mob(sw0)
    q_well = prod.well_index * (mw + mo)[c] * (p1[c] - prod.control_value * 1e6)
    fo = mo[c] / (mw[c] + mo[c] + 1e-10)
    np.testing.assert_allclose(float(rates[0]), float(q_well * fo * 86400.0), rtol=1e-9)


def test_autograd_matches_central_differences():
    cfg, f, dt, model = _case()
    _, f2 = scenarios.adjoint_case(seed=5, nx=16, ny=16, nz=2, steps=3)
    target = oadj.producer_rates(model(dict(f2, poro=f["poro"])), dt, 3).numpy()
    J, g_lnk, g_poro, _ = oadj.objective(model(), dt, 3, target)
    assert J > 0
    t = oadj.TorchIMPES(model())
    rng = np.random.default_rng(0)
    tgt = torch.tensor(target)

    def J_of(lnk, poro):
        return float(((oadj.producer_rates(model(), dt, 3, lnk, poro) - tgt) ** 2).sum())
    for c in rng.choice(t.lnk0.numel(), 5, replace=False):
        h = 1e-4
        lk = t.lnk0.clone(); lk[c] += h
        jp = J_of(lk, t.poro0)
        lk[c] -= 2 * h
        jm = J_of(lk, t.poro0)
        assert (jp - jm) / (2 * h) == pytest.approx(g_lnk[c], rel=2e-3, abs=1e-6 * np.abs(g_lnk).max())
        hp = 1e-4 * float(t.poro0[c])
        po = t.poro0.clone(); po[c] += hp
        jp = J_of(t.lnk0, po)
        po[c] -= 2 * hp
        jm = J_of(t.lnk0, po)
        assert (jp - jm) / (2 * hp) == pytest.approx(g_poro[c], rel=2e-3, abs=1e-6 * np.abs(g_poro).max())


def test_oracle_adjoint_matches_autograd_through_the_reference(golden):
    """The dense restatement's objective, rates and gradients against autograd
    through the reference's own IMPES step with a dense pressure solve on the
    16x16x2 sub-case, 6 steps (fixture made by make_golden.py --adjoint-only)."""
    import json
    g = golden("adjoint_ref_16x16x2")
    m = Model(json.loads(str(g["cfg"])), g["kx"], g["ky"], g["kz"], g["poro"])
    J, g_lnk, g_poro, q = oadj.objective(m, float(g["dt"]), int(g["steps"]), g["target"])
    assert J == pytest.approx(float(g["J"]), rel=1e-10)
    np.testing.assert_allclose(q, g["rates"], rtol=1e-10)
    assert np.linalg.norm(g_lnk - g["g_lnk"]) <= 1e-10 * np.linalg.norm(g["g_lnk"])
    assert np.linalg.norm(g_poro - g["g_poro"]) <= 1e-10 * np.linalg.norm(g["g_poro"])
