"""K1 pressure assembly and K4 saturation update on the GPU against the oracle
and the reference's recorded outputs."""
import numpy as np
import pytest
import torch

from gpu_util import cfg_fields, gpu_sim, oracle_model, rel_max, to_np

pytestmark = pytest.mark.gpu

CASES = ["two_phase_32x32", "two_phase_64x64", "two_phase_16x16x2", "black_oil_10x10x4",
         "gas_injection_12x12x3", "three_phase_16x16x3"]


@pytest.mark.parametrize("name", CASES)
def test_assembly_matches_reference_step1(golden, name):
    """Pattern and well cells bit-exact; values and RHS of the reference's first
    pressure system to 1e-13 (max-norm relative)."""
    g = golden(name)
    cfg, f = cfg_fields(g)
    _, fl, wm, sim = gpu_sim(cfg, f)
    rowptr, col, val, rhs = sim.assemble(float(g["dt"]))
    assert np.array_equal(to_np(rowptr), g["A0_crow"])
    assert np.array_equal(to_np(col), g["A0_col"])
    assert rel_max(to_np(val), g["A0_val"]) <= 1e-13
    assert rel_max(to_np(rhs), g["b0"]) <= 1e-13
    wells = wm.get_wells()
    assert [w.cell_index_flat for w in wells] == list(g["well_cells"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("seed", [0, 1])
def test_assembly_random_states_vs_oracle(golden, name, seed):
    """Perturbed p/Sw/Sg (mixed upwind directions, mobile gas, capillarity)."""
    g = golden(name)
    cfg, f = cfg_fields(g)
    m = oracle_model(g)
    rng = np.random.default_rng(seed)
    m.p = m.p * (1.0 + 0.05 * rng.standard_normal(m.N))
    m.sw = np.clip(0.2 + 0.5 * rng.random(m.N), 0.2, 0.8)
    m.sg = np.clip(0.3 * rng.random(m.N) * (m.pvt is not None), 0.0, 0.8 - m.sw)
    A, b, _ = m.assemble(float(g["dt"]))
    _, fl, _, sim = gpu_sim(cfg, f)
    dev = fl.pressure.device
    _, _, val, rhs = sim.assemble(float(g["dt"]), p=torch.tensor(m.p, device=dev),
                                  s_w=torch.tensor(m.sw, device=dev), s_g=torch.tensor(m.sg, device=dev))
    assert rel_max(to_np(val), A.data) <= 1e-12
    assert rel_max(to_np(rhs), b) <= 1e-12


@pytest.mark.parametrize("name", CASES)
def test_saturation_matches_reference_step1(golden, name):
    """Given the reference's first pressure, Sw/Sg to 1e-12 and the balances."""
    g = golden(name)
    cfg, f = cfg_fields(g)
    m = oracle_model(g)
    dt = float(g["dt"])
    p1 = g["p"][0]
    n_ref = m.saturation(p1.copy(), dt)
    _, fl, _, sim = gpu_sim(cfg, f)
    n = sim.saturation(torch.tensor(p1, device=fl.pressure.device), dt)
    assert n == n_ref
    assert np.abs(to_np(fl.s_w) - g["sw"][0]).max() <= 1e-12
    assert np.abs(to_np(fl.s_g) - g["sg"][0]).max() <= 1e-12
    so = to_np(fl.s_o)
    assert np.abs(so - (1.0 - to_np(fl.s_w) - to_np(fl.s_g))).max() <= 1e-15
    mb = sim.mass_balance
    ref = g["balances"][0]
    got = [mb[ph][io] for ph in ("water", "oil", "gas") for io in ("in", "out")]
    assert np.allclose(got, ref[:6], rtol=1e-10, atol=1e-300)
    cb = sim.component_balance
    gotc = [cb[c][k] for c in ("oil", "gas") for k in ("in", "out", "accum")]
    assert np.allclose(gotc, ref[6:], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", ["black_oil_10x10x4", "gas_injection_12x12x3", "two_phase_16x16x2"])
def test_saturation_random_states_vs_oracle(golden, name):
    g = golden(name)
    cfg, f = cfg_fields(g)
    m = oracle_model(g)
    rng = np.random.default_rng(5)
    m.sw = np.clip(0.2 + 0.4 * rng.random(m.N), 0.2, 0.8)
    m.sg = np.clip(0.2 * rng.random(m.N) * (m.pvt is not None), 0.0, 0.8 - m.sw)
    sw0, sg0 = m.sw.copy(), m.sg.copy()
    p_new = g["p"][0] * (1.0 + 0.01 * rng.standard_normal(m.N))
    dt = float(g["dt"])
    n_ref = m.saturation(p_new.copy(), dt)
    _, fl, _, sim = gpu_sim(cfg, f)
    dev = fl.pressure.device
    fl.s_w = torch.tensor(sw0, device=dev).reshape(fl.s_w.shape)
    fl.s_g = torch.tensor(sg0, device=dev).reshape(fl.s_g.shape)
    n = sim.saturation(torch.tensor(p_new, device=dev), dt)
    assert n == n_ref
    assert np.abs(to_np(fl.s_w) - m.sw).max() <= 1e-11
    assert np.abs(to_np(fl.s_g) - m.sg).max() <= 1e-11


def test_transmissibility_and_pore_volume(golden):
    g = golden("black_oil_10x10x4")
    cfg, f = cfg_fields(g)
    m = oracle_model(g)
    _, _, _, sim = gpu_sim(cfg, f)
    tx, ty, tz, pv = sim.static_fields()
    assert np.array_equal(to_np(tx), m.Tx.ravel())
    assert np.array_equal(to_np(ty), m.Ty.ravel())
    assert np.array_equal(to_np(tz), m.Tz.ravel())
    assert np.array_equal(to_np(pv), m.pv)
