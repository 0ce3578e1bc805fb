"""The host layer's translation of a reference-schema config into the C ABI's
model and well descriptors, checked field by field against the oracle's own
parse of the same config, for every recorded fixture.  Runs on the CPU: the
package's Reservoir and Fluid are built on CPU tensors here by patching the
device resolver of the module under test (the product path itself refuses
anything but CUDA)."""
import json

import pytest
import torch

from oracle.impes import Model

CASES = ["two_phase_32x32", "two_phase_64x64", "two_phase_16x16x2", "black_oil_10x10x4",
         "gas_injection_12x12x3", "three_phase_16x16x3", "wells_surface_oil_6x6",
         "wells_surface_gas_6x6", "wells_rv_liquid_6x6", "wells_surface_water_6x6",
         "cg_two_phase_20x16x2", "cg_three_phase_16x16x3"]


@pytest.fixture
def sim_module(monkeypatch):
    from impes_b200 import simulator
    monkeypatch.setattr(simulator, "_cuda_device", lambda device=None: torch.device("cpu"))
    return simulator


@pytest.mark.parametrize("name", CASES)
def test_model_descriptor_matches_oracle_parse(golden, sim_module, name):
    g = golden(name)
    cfg = json.loads(str(g["cfg"]))
    res = sim_module.Reservoir(cfg["reservoir"])
    fl = sim_module.Fluid(cfg["fluid"], res)
    d = sim_module.model_desc(res, fl, cfg["simulation"])
    m = Model(cfg, g["kx"], g["ky"], g["kz"], g["poro"])
    assert (d.nx, d.ny, d.nz) == (m.nx, m.ny, m.nz)
    assert (d.dx, d.dy, d.dz) == (m.dx, m.dy, m.dz)
    assert (d.mu_o, d.mu_w, d.mu_g) == (m.mu_oil, m.mu_water, m.mu_gas)
    assert (d.rho_o_ref, d.rho_w_ref, d.rho_g_ref) == (m.rho_oil_ref, m.rho_water_ref, m.rho_gas_ref)
    assert (d.c_o, d.c_w, d.c_g, d.c_r) == (m.c_o, m.c_w, m.c_g, m.c_r)
    assert d.cf == m.cf
    assert d.relperm_model == (1 if m.relperm_model == "stone2" else 0)
    assert (d.nw, d.no, d.ng, d.now, d.nog) == tuple(float(v) for v in (m.nw, m.no, m.ng, m.now, m.nog))
    assert (d.ko_end_w, d.ko_end_g) == (m.ko_end_w, m.ko_end_g)
    assert (d.sw_cr, d.so_r, d.sg_cr) == (m.sw_cr, m.so_r, m.sg_cr)
    assert (d.pc_scale, d.pc_exponent) == (float(m.pc_scale), float(m.pc_exponent))
    assert (d.pc_og_scale, d.pc_og_exponent) == (float(m.pc_og_scale), float(m.pc_og_exponent))
    sp = m.sim_params
    assert d.global_rate_scale == float(sp.get("global_rate_scale", 1.0))
    assert d.max_saturation_change == float(sp.get("max_saturation_change", 0.05))
    assert d.max_substeps == int(sp.get("max_substeps", 20))
    assert d.pvt_rows == (0 if m.pvt is None else len(m.pvt.P))
    # initial state as the oracle sets it
    assert float(fl.pressure.reshape(-1)[0]) == m.p[0]
    assert float(fl.s_w.reshape(-1)[0]) == m.sw[0] and float(fl.s_g.reshape(-1)[0]) == m.sg[0]


@pytest.mark.parametrize("name", CASES)
def test_well_descriptors_match_oracle_parse(golden, sim_module, name):
    g = golden(name)
    cfg = json.loads(str(g["cfg"]))
    res = sim_module.Reservoir(cfg["reservoir"])
    wells = sim_module.WellManager(cfg["wells"], res).get_wells()
    arr = sim_module.well_descs(wells)
    m = Model(cfg, g["kx"], g["ky"], g["kz"], g["poro"])
    assert len(wells) == len(m.wells)
    for n, (d, w) in enumerate(zip(arr, m.wells)):
        assert (d.i, d.j, d.k) == (w.i, w.j, w.k)
        assert d.is_injector == (w.type == "injector")
        assert d.control_bhp == (w.control_type == "bhp")
        assert d.value == float(w.control_value)
        assert d.well_index == w.well_index
        assert d.injected_phase == (1 if w.injected_phase == "gas" else 0)
        assert d.surface_rate == (1 if w.rate_type == "surface" else 0)
        assert d.surface_phase == {"oil": 0, "water": 1, "gas": 2, "liquid": 3}[(w.surface_phase or "liquid").lower()]
        lims = w.limits or {}
        for q, (key, bit) in enumerate((("wopr", 1), ("wlpr", 2), ("wgpr", 4), ("liqr", 8))):
            assert bool(d.limit_mask & bit) == (key in lims)
            if key in lims:
                assert d.limits[q] == float(lims[key])
        assert d.has_bhp_min == (w.bhp_min is not None)
        if w.bhp_min is not None:
            assert d.bhp_min == float(w.bhp_min)
    # the flat cell index the step uses (simulation.py:1629-1630)
    assert [(w.i * res.ny + w.j) * res.nz + w.k for w in wells] == list(g["well_cells"])


def test_matrix_conversion_follows_the_reference_coalesce_then_cast():
    """to_csr32 against _to_csr_double's steps (pressure_amg.py:11-32):
    duplicates of a COO input are summed in the input's dtype by coalesce(), the
    CSR is cast to float64 afterwards; dense inputs drop their zeros; scipy
    inputs of any format sum duplicates and sort columns without touching the
    caller's matrix; a (rowptr, col, val, shape) tuple passes through."""
    import numpy as np
    import scipy.sparse as sp
    from impes_b200.amg import to_csr32
    cpu = torch.device("cpu")
    rng = np.random.default_rng(4)
    n, m = 40, 300
    r = torch.tensor(rng.integers(0, n, m)); c = torch.tensor(rng.integers(0, n, m))
    v = torch.tensor(rng.standard_normal(m), dtype=torch.float32)
    A = torch.sparse_coo_tensor(torch.stack([r, c]), v, (n, n))
    ref = A.coalesce().to_sparse_csr()
    rowptr, col, val, shape = to_csr32(A, cpu)
    assert shape == (n, n) and rowptr.dtype == torch.int32 and col.dtype == torch.int32
    assert torch.equal(rowptr, ref.crow_indices().int()) and torch.equal(col, ref.col_indices().int())
    assert val.dtype == torch.float64 and torch.equal(val, ref.values().double())
    # same matrix given as CSR
    r2 = to_csr32(ref, cpu)
    assert all(torch.equal(a, b) for a, b in zip(r2[:3], (rowptr, col, val)))
    # dense input: explicit zeros are not stored
    D = torch.zeros(n, n, dtype=torch.float64)
    D[3, 5], D[7, 7], D[39, 0] = 1.5, -2.0, 0.25
    rp, cl, vl, _ = to_csr32(D, cpu)
    assert vl.tolist() == [1.5, -2.0, 0.25] and cl.tolist() == [5, 7, 0]
    assert rp[-1].item() == 3
    # scipy COO with duplicates
    S = sp.coo_matrix((v.double().numpy(), (r.numpy(), c.numpy())), shape=(n, n))
    rp, cl, vl, _ = to_csr32(S, cpu)
    T = S.tocsr(); T.sum_duplicates(); T.sort_indices()
    assert np.array_equal(rp.numpy(), T.indptr) and np.array_equal(cl.numpy(), T.indices)
    assert np.array_equal(vl.numpy(), T.data)
    # scipy CSR with unsorted and repeated columns: summed and sorted in a copy
    U = sp.csr_matrix((np.array([1.0, 2.0, 4.0, 8.0]), np.array([3, 1, 3, 0]), np.array([0, 3, 4])),
                      shape=(2, 4))
    before = (U.indices.copy(), U.data.copy())
    rp, cl, vl, _ = to_csr32(U, cpu)
    assert rp.tolist() == [0, 2, 3] and cl.tolist() == [1, 3, 0] and vl.tolist() == [2.0, 5.0, 8.0]
    assert np.array_equal(U.indices, before[0]) and np.array_equal(U.data, before[1])
    # pass-through
    tup = (rowptr, col, val, shape)
    assert to_csr32(tup, cpu) is tup


@pytest.mark.parametrize("source", ["pvt_path", "pvt.path", "pvt.table"])
def test_pvt_sources_give_the_same_table(sim_module, tmp_path, source):
    """fluid.py:52-58: a PVT table given by ``pvt_path``, by ``pvt.path`` or
    inline as ``pvt.table`` packs to the same rows for the C ABI and evaluates
    like the oracle's table (np.interp with flat ends, pvt.py:48-64)."""
    import numpy as np
    from impes_b200 import scenarios
    from oracle.impes import PVT
    table = scenarios.pvt_table_black_oil(rv_max=2.0e-4)
    path = tmp_path / "pvt.json"
    path.write_text(json.dumps(table))
    fluid_cfg = {"pressure": 20.0, "s_w": 0.2, "s_g": 0.0}
    fluid_cfg.update({"pvt_path": {"pvt_path": str(path)}, "pvt.path": {"pvt": {"path": str(path)}},
                      "pvt.table": {"pvt": {"table": table}}}[source])
    res = sim_module.Reservoir({"dimensions": [2, 2, 1]})
    fl = sim_module.Fluid(fluid_cfg, res)
    packed = fl.pvt.packed()
    assert packed.shape == (20, 9)
    ref = PVT(table)
    cols = ("Bo", "Bw", "Bg", "mu_o", "mu_w", "mu_g", "Rs", "Rv")
    np.testing.assert_array_equal(packed[:, 0], ref.P)
    for q, key in enumerate(cols, start=1):
        np.testing.assert_array_equal(packed[:, q], ref.cols[key])
    p_mpa = np.array([1.0, 5.0, 12.345, 27.5, 40.0, 60.0])
    ours = fl.pvt.eval(p_mpa)
    for key in cols:
        np.testing.assert_array_equal(ours[key], ref.eval(p_mpa * 1e6, key))


def test_alternative_well_and_capillary_schemas(sim_module):
    """well.py:77-92 accepts wells as coordinates/control or as i, j, k /
    control_type, control_value; fluid.py:97-105 accepts capillarity as a
    capillary_pressure section or as top-level keys.  Both forms give the same
    descriptors."""
    res = sim_module.Reservoir({"dimensions": [6, 5, 3]})
    flat = [{"name": "I", "type": "injector", "i": 1, "j": 2, "k": 0, "radius": 0.1,
             "control_type": "rate", "control_value": 40.0, "injected_phase": "water"},
            {"name": "P", "type": "producer", "i": 4, "j": 3, "k": 2, "radius": 0.12,
             "control_type": "bhp", "control_value": 15.0}]
    nested = [{"name": "I", "type": "injector", "coordinates": [1, 2, 0], "radius": 0.1,
               "control": {"type": "rate", "value": 40.0}, "injected_phase": "water"},
              {"name": "P", "type": "producer", "coordinates": [4, 3, 2], "radius": 0.12,
               "control": {"type": "bhp", "value": 15.0}}]
    a = sim_module.well_descs(sim_module.WellManager(flat, res).get_wells())
    b = sim_module.well_descs(sim_module.WellManager(nested, res).get_wells())
    fields = [name for name, _ in a[0]._fields_ if name != "limits"]
    for x, y in zip(a, b):
        assert [getattr(x, f) for f in fields] == [getattr(y, f) for f in fields]
    with pytest.raises(ValueError):
        sim_module.WellManager([{"name": "X", "type": "producer", "radius": 0.1,
                                 "control_type": "bhp", "control_value": 1.0}], res)
    sect = sim_module.Fluid({"capillary_pressure": {"pc_scale": 3.0e4, "pc_exponent": 0.7}}, res)
    top = sim_module.Fluid({"pc_scale": 3.0e4, "pc_exponent": 0.7}, res)
    da, db = sim_module.model_desc(res, sect, {}), sim_module.model_desc(res, top, {})
    assert (da.pc_scale, da.pc_exponent) == (db.pc_scale, db.pc_exponent) == (3.0e4, 0.7)


def test_apply_reference_fix_pins_one_dof():
    """_apply_reference_fix (classical_amg.py:660-686): the anchor's row and
    column are dropped and its diagonal becomes 1, added when the matrix has no
    stored diagonal there; every other entry is kept, including explicit
    zeros."""
    import numpy as np
    import scipy.sparse as sp
    from impes_b200.amg import _apply_reference_fix
    from test_oracle_pin import laplacian_2d, pin
    A = laplacian_2d(5)
    for k in (0, 7, 24):
        T = torch.sparse_csr_tensor(torch.tensor(A.indptr), torch.tensor(A.indices), torch.tensor(A.data),
                                    size=A.shape)
        F = _apply_reference_fix(T, k)
        got = sp.csr_matrix((F.values().numpy(), F.col_indices().numpy(), F.crow_indices().numpy()), shape=A.shape)
        assert abs(got - pin(A, k)).max() == 0.0
    # no stored diagonal at the anchor, and an explicit zero elsewhere
    r = torch.tensor([[0, 0, 1, 1, 1, 2, 2], [1, 2, 0, 1, 2, 2, 1]])
    v = torch.tensor([-1.0, 0.0, -1.0, 0.0, -2.0, 3.0, 0.5], dtype=torch.float64)
    T = torch.sparse_coo_tensor(r, v, (3, 3)).coalesce().to_sparse_csr()
    Fs = _apply_reference_fix(T, 0)
    F = Fs.to_dense().numpy()
    np.testing.assert_array_equal(F, [[1.0, 0.0, 0.0], [0.0, 0.0, -2.0], [0.0, 0.5, 3.0]])
    assert F.dtype == np.float64
    # stored pattern: (0,0) added, (1,1) kept as an explicit zero, row/column 0 dropped
    pattern = list(zip(np.repeat(np.arange(3), np.diff(Fs.crow_indices().numpy())), Fs.col_indices().tolist()))
    assert pattern == [(0, 0), (1, 1), (1, 2), (2, 1), (2, 2)]
