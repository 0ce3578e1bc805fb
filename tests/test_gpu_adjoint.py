"""The CUDA adjoint against autograd through the dense float64 restatement of the
step (16x16x2) and against central differences of the GPU forward run at the
full 64x64x8, 50-step size."""
import numpy as np
import pytest
import torch

from impes_b200 import scenarios
from oracle import adjoint as oadj
from oracle.impes import Model

pytestmark = pytest.mark.gpu

SMALL = dict(nx=16, ny=16, nz=2)


def _small(steps, seed=3, target_seed=5):
    cfg, f = scenarios.adjoint_case(seed=seed, steps=steps, **SMALL)
    _, f2 = scenarios.adjoint_case(seed=target_seed, steps=steps, **SMALL)
    dt = cfg["simulation"]["time_step_days"] * 86400.0
    m_tgt = Model(cfg, f2["kx"], f2["ky"], f2["kz"], f["poro"])
    target = oadj.producer_rates(m_tgt, dt, steps).numpy()
    return cfg, f, dt, target


def test_rates_match_dense_restatement():
    from impes_b200.adjoint import producer_rates
    cfg, f, dt, _ = _small(6)
    got = producer_rates(cfg, f, 6, dt, tol=1e-13)
    ref = oadj.producer_rates(Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"]), dt, 6).numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-8)


@pytest.mark.parametrize("ckpt", [2, 0])
def test_gradient_matches_autograd(ckpt):
    from impes_b200.adjoint import misfit_gradient
    steps = 6
    cfg, f, dt, target = _small(steps)
    J, g_lnk, g_poro, q = oadj.objective(Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"]), dt, steps, target)
    out = misfit_gradient(cfg, f, target, steps, dt, checkpoint_every=ckpt, tol=1e-13, adjoint_tol=1e-13)
    assert out["J"] == pytest.approx(J, rel=1e-8)
    np.testing.assert_allclose(out["rates"], q, rtol=1e-8)
    gl = out["g_lnk"].reshape(-1).cpu().numpy()
    gp = out["g_poro"].reshape(-1).cpu().numpy()
    assert np.linalg.norm(gl - g_lnk) <= 1e-6 * np.linalg.norm(g_lnk)
    assert np.linalg.norm(gp - g_poro) <= 1e-6 * np.linalg.norm(g_poro)
    st = out["stats"]
    assert st["checkpoints"] == (3 if ckpt == 2 else 1)
    assert st["recomputed_steps"] == (4 if ckpt == 2 else 0)


def test_autograd_function_backward():
    from impes_b200.adjoint import misfit, misfit_gradient
    steps = 4
    cfg, f, dt, target = _small(steps)
    lnk = torch.log(torch.tensor(f["kx"], device="cuda")).requires_grad_(True)
    poro = torch.tensor(f["poro"], device="cuda").requires_grad_(True)
    J = misfit(lnk, poro, cfg, target, steps, dt, tol=1e-13, adjoint_tol=1e-13)
    (3.0 * J).backward()
    # the direct call gets kx itself rather than exp(log(kx)): last-bit input differences
    out = misfit_gradient(cfg, f, target, steps, dt, tol=1e-13, adjoint_tol=1e-13)
    assert float(J.detach()) == pytest.approx(out["J"], rel=1e-8)
    torch.testing.assert_close(lnk.grad, 3.0 * out["g_lnk"], rtol=1e-6, atol=1e-9 * float(out["g_lnk"].abs().max()))
    torch.testing.assert_close(poro.grad, 3.0 * out["g_poro"], rtol=1e-6, atol=1e-9 * float(out["g_poro"].abs().max()))


def test_refuses_models_outside_scope():
    from impes_b200 import _lib
    from impes_b200.adjoint import misfit_gradient
    cfg, f = scenarios.black_oil_5spot(nx=6, ny=6, nz=2, steps=2)
    with pytest.raises(_lib.ImpesError, match="outside its scope|Corey"):
        misfit_gradient(cfg, f, np.zeros((2, 1)), 2)


def test_full_size_gradient_vs_central_differences():
    """64x64x8, 50 steps of 2 days, checkpoints every 10: the adjoint gradient
    against central differences of the GPU forward run on 20 random cells
    (ln k, h = 1e-4) and 8 cells (porosity, relative h = 1e-3).  J (~200) carries
    ~1e-9 relative noise from the iterative pressure solves, so smaller steps
    measure the noise."""
    from impes_b200.adjoint import misfit_gradient, producer_rates
    steps = 50
    cfg, f = scenarios.adjoint_case(seed=3, steps=steps)
    _, f2 = scenarios.adjoint_case(seed=5, steps=steps)
    dt = cfg["simulation"]["time_step_days"] * 86400.0
    target = producer_rates(cfg, dict(f2, poro=f["poro"]), steps, dt, tol=1e-13)
    out = misfit_gradient(cfg, f, target, steps, dt, checkpoint_every=10, tol=1e-13, adjoint_tol=1e-12)
    gl = out["g_lnk"].reshape(-1).cpu().numpy()
    gp = out["g_poro"].reshape(-1).cpu().numpy()
    assert out["stats"]["checkpoints"] == 5 and out["stats"]["recomputed_steps"] == 40

    def J(fields):
        q = producer_rates(cfg, fields, steps, dt, tol=1e-13)
        return float(((q - target) ** 2).sum())
    rng = np.random.default_rng(7)
    lnk = np.log(f["kx"]).reshape(-1)
    rel_k = []
    for c in rng.choice(lnk.size, 20, replace=False):
        h = 1e-4
        vals = []
        for s in (1, -1):
            l2 = lnk.copy(); l2[c] += s * h
            kx = np.exp(l2).reshape(f["kx"].shape)
            vals.append(J(dict(kx=kx, ky=kx, kz=kx, poro=f["poro"])))
        fd = (vals[0] - vals[1]) / (2 * h)
        rel_k.append(abs(fd - gl[c]) / max(abs(gl[c]), 1e-3 * np.abs(gl).max()))
    rel_p = []
    poro = f["poro"].reshape(-1)
    for c in rng.choice(poro.size, 8, replace=False):
        h = 1e-3 * poro[c]
        vals = []
        for s in (1, -1):
            p2 = poro.copy(); p2[c] += s * h
            vals.append(J(dict(f, poro=p2.reshape(f["poro"].shape))))
        fd = (vals[0] - vals[1]) / (2 * h)
        rel_p.append(abs(fd - gp[c]) / max(abs(gp[c]), 1e-3 * np.abs(gp).max()))
    rel_k, rel_p = np.array(rel_k), np.array(rel_p)
    print("ln k FD relative errors:", np.sort(rel_k))
    print("porosity FD relative errors:", np.sort(rel_p))
    assert np.median(rel_k) < 1e-3 and np.mean(rel_k < 1e-2) >= 0.9
    assert np.median(rel_p) < 1e-3 and np.mean(rel_p < 1e-2) >= 0.9
