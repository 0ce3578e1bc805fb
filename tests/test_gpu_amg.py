"""AMG setup, V-cycle, stand-alone solve, update and FGMRES on the GPU vs the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from gpu_util import csr_from, to_np
from oracle import amg as oa
from test_oracle_pin import laplacian_2d, pin

pytestmark = pytest.mark.gpu


def gpu_amg(A, **kw):
    from impes_b200.amg import ClassicalAMG
    return ClassicalAMG(A, **kw)


# ClassicalAMG hierarchies the reference built (fixture) and the trajectory whose
# recorded matrices they were built from: a 2-D two-phase matrix and two 3-D
# ones (black oil with PVT, gravity and capillarity; three phases without PVT)
AMG_FIXTURES = [("amg_two_phase_32x32", "two_phase_32x32"),
                ("amg_black_oil_10x10x4", "black_oil_10x10x4"),
                ("amg_three_phase_16x16x3", "three_phase_16x16x3")]


@pytest.fixture(scope="module", params=AMG_FIXTURES, ids=[a for a, _ in AMG_FIXTURES])
def case(golden, request):
    amg_name, traj_name = request.param
    g = golden(amg_name)
    t = golden(traj_name)
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    A2 = sp.csr_matrix((t["A_val_all"][1], t["A0_col"], t["A0_crow"]), shape=(n, n))
    return g, t, A, A2


def compare_hierarchy(amg, ref, pval_rtol=1e-7):
    levels = amg.levels
    assert [lv["n"] for lv in levels] == [lv["n"] for lv in ref.levels]
    for lv, rl in zip(levels, ref.levels):
        Ag = csr_from(lv["A"].crow_indices(), lv["A"].col_indices(), lv["A"].values(), lv["n"])
        Ar = rl["A"]
        assert abs(Ag - Ar).max() <= 1e-8 * abs(Ar).max()
        np.testing.assert_allclose(to_np(lv["inv_relax"]), rl["inv_relax"], rtol=1e-7)
        if rl["P"] is not None:
            P = lv["P"]
            assert np.array_equal(to_np(P.crow_indices()), rl["P"].indptr)
            assert np.array_equal(to_np(P.col_indices()), rl["P"].indices)
            np.testing.assert_allclose(to_np(P.values()), rl["P"].data, rtol=pval_rtol, atol=1e-9)


def test_hierarchy_matches_reference_fixture(case):
    """Same tie-break stream as the reference run -> same levels, same P patterns."""
    g, t, A, _ = case
    amg = gpu_amg(A, coarsest_size=int(g["coarsest"]), seed=int(g["seed"]))
    assert [lv["n"] for lv in amg.levels] == [int(len(g[f"L{l}_inv_relax"])) for l in range(int(g["n_levels"]))]
    for l, lv in enumerate(amg.levels):
        if not lv["is_coarsest"]:
            assert np.array_equal(to_np(lv["P"].crow_indices()), g[f"L{l}_P_crow"])
            assert np.array_equal(to_np(lv["P"].col_indices()), g[f"L{l}_P_col"])
            np.testing.assert_allclose(to_np(lv["P"].values()), g[f"L{l}_P_val"], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(to_np(amg.Dhalf_inv), g["Dhalf_inv"], rtol=1e-14)


def test_vcycle_solve_apply_update_vs_oracle(case):
    g, t, A, A2 = case
    seed, cs = int(g["seed"]), int(g["coarsest"])
    amg = gpu_amg(A, coarsest_size=cs, seed=seed)
    ref = oa.AMG(A, coarsest_size=cs, seed=seed)
    compare_hierarchy(amg, ref)
    b = g["b"]
    bs = ref.Dhalf_inv * b
    v_ref = ref.vcycle(0, np.zeros_like(bs), bs)
    v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda")))
    assert np.linalg.norm(v - v_ref) <= 1e-9 * np.linalg.norm(v_ref)
    x_ref, cyc_ref, _ = ref.solve(b, tol=1e-30, max_iter=4)
    x = to_np(amg.solve(torch.tensor(b, device="cuda"), tol=1e-30, max_iter=4))
    assert amg.last_stats["cycles"] == cyc_ref == 4
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    # against the reference's own V-cycle output recorded in the fixture
    assert np.linalg.norm(x - g["solve_x"]) <= 1e-8 * np.linalg.norm(g["solve_x"])
    xa = to_np(amg.apply(torch.tensor(b, device="cuda"), cycles=2))
    assert np.linalg.norm(xa - g["apply_x"]) <= 1e-8 * np.linalg.norm(g["apply_x"])
    amg.update_matrix(A2)
    ref.update_matrix(A2)
    compare_hierarchy(amg, ref)
    x2 = to_np(amg.solve(torch.tensor(g["b2"], device="cuda"), tol=1e-30, max_iter=3))
    assert np.linalg.norm(x2 - g["update_solve_x"]) <= 1e-8 * np.linalg.norm(g["update_solve_x"])


def test_laplacian_quality_kat():
    """The reference's AMG KAT (tests/test_amg_pressure_solver.py:89-106)."""
    A = pin(laplacian_2d(12), 0)
    amg = gpu_amg(A, theta=0.25, max_levels=10, coarsest_size=40)
    n = A.shape[0]
    rng = np.random.default_rng(0)
    for v in (np.ones(n), np.linspace(0, 1, n), rng.standard_normal(n)):
        v = v / np.linalg.norm(v)
        z = to_np(amg.apply(torch.tensor(v, device="cuda"), cycles=3))
        assert np.linalg.norm(A @ z - v) / np.linalg.norm(v) < 5e-2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("norm", ["jacobi", "equilibrated"])
def test_fgmres_reaches_direct_solution(golden, precision, norm):
    t = golden("two_phase_64x64")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    b = t["b0"]
    x_direct = spla.spsolve(A.tocsc(), b)
    amg = gpu_amg(A, coarsest_size=200, seed=1)
    # the equilibrated norm is dominated by the BHP-well row (its relative
    # residual bottoms out near 3e-16), so it cannot certify as tight a solution
    tol, bound = (1e-13, 1e-9) if norm == "jacobi" else (1e-15, 1e-5)
    x, st = amg.fgmres(torch.tensor(b, device="cuda"), tol=tol, restart=40, max_iters=300, norm=norm,
                       precision=precision)
    x = to_np(x)
    assert st["converged"], st
    assert np.abs(x - x_direct).max() <= bound * np.abs(x_direct).max(), st


def test_fgmres_respects_iteration_cap(golden):
    t = golden("two_phase_64x64")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = gpu_amg(A, coarsest_size=200)
    _, st = amg.fgmres(torch.tensor(t["b0"], device="cuda"), tol=1e-30, restart=10, max_iters=7)
    assert st["iterations"] == 7 and not st["converged"]


def test_setup_rejects_bad_csr():
    from impes_b200._lib import ImpesError
    rowptr = torch.tensor([0, 2, 3], dtype=torch.int32, device="cuda")
    col = torch.tensor([1, 0, 5], dtype=torch.int32, device="cuda")   # column out of range
    val = torch.ones(3, dtype=torch.float64, device="cuda")
    with pytest.raises(ImpesError):
        gpu_amg((rowptr, col, val, (2, 2)))
    val = torch.tensor([1.0, float("nan"), 1.0], dtype=torch.float64, device="cuda")
    col = torch.tensor([0, 1, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(ImpesError):
        gpu_amg((rowptr, col, val, (2, 2)))


def test_setup_is_deterministic(golden):
    t = golden("two_phase_64x64")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    a1, a2 = gpu_amg(A, coarsest_size=100, seed=3), gpu_amg(A, coarsest_size=100, seed=3)
    for l1, l2 in zip(a1.levels, a2.levels):
        assert torch.equal(l1["A"].values(), l2["A"].values())
    b = torch.tensor(t["b0"], device="cuda")
    assert torch.equal(a1.fgmres(b, tol=1e-10)[0], a2.fgmres(b, tol=1e-10)[0])


def test_larger_3d_hierarchy_vs_oracle():
    """20x20x10 black-oil-like matrix: same structure as the oracle hierarchy."""
    from impes_b200 import scenarios
    from oracle.impes import Model
    cfg, f = scenarios.black_oil_5spot(seed=1, nx=20, ny=20, nz=10, inj_rate=50.0)
    m = Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"], pvt_table=f["pvt"])
    A, b, _ = m.assemble(5 * 86400.0)
    amg = gpu_amg(A, coarsest_size=200, seed=2)
    ref = oa.AMG(A, coarsest_size=200, seed=2)
    compare_hierarchy(amg, ref, pval_rtol=1e-6)


def test_graph_replay_matches_direct_launches(golden, monkeypatch):
    """V-cycles replayed from CUDA graphs give bitwise the same FGMRES iterates as
    direct launches (IMPES_NO_GRAPHS=1 is read at setup)."""
    t = golden("two_phase_64x64")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    b = torch.tensor(t["b0"], device="cuda")
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("IMPES_NO_GRAPHS", flag)
        amg = gpu_amg(A, coarsest_size=100, seed=3)
        for prec in ("fp64", "mixed"):
            outs.append(amg.fgmres(b, tol=1e-10, precision=prec)[0])
        outs.append(amg.solve(b, tol=1e-30, max_iter=3))
    for a, c in zip(outs[:3], outs[3:]):
        assert torch.equal(a, c)


def test_phase_timers_inside_graphs(golden):
    from impes_b200 import _lib
    t = golden("two_phase_64x64")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = gpu_amg(A, coarsest_size=100)
    _lib.timing_enable(True)
    _lib.timing_collect()
    _, st = amg.fgmres(torch.tensor(t["b0"], device="cuda"), tol=1e-8, precision="mixed")
    ph = _lib.timing_collect()
    _lib.timing_enable(False)
    assert ph["vcycle"][0] == st["iterations"]
    assert ph["smooth_l0"][0] >= 4 * st["iterations"] and ph["smooth_l0"][1] > 0


def test_mixed_vcycle_on_wide_levels_matches_fp64():
    """A hierarchy (640,000 cells) whose coarse levels have rows of more than 512
    entries and more than 48 MB of values and columns (the fp32 sweep streams
    those through shared memory), updated through the fp32 Galerkin chain: one
    fp32 V-cycle agrees with the fp64 one to fp32 rounding, and the fp64 levels
    exported afterwards are those of the updated matrix."""
    from impes_b200 import scenarios
    from impes_b200.simulator import build_from_config
    cfg, f = scenarios.gas_injection_1m(seed=2, nx=160, ny=160, nz=25)
    _, fl, _, sim = build_from_config(cfg, f, device="cuda")
    rowptr, col, val, rhs = sim.assemble(2 * 86400.0)
    n = rhs.numel()
    A = torch.sparse_csr_tensor(rowptr.long(), col.long(), val, size=(n, n))
    amg = gpu_amg(A, theta=0.2, max_levels=20, coarsest_size=120, mixed_precision=True)
    rng = np.random.default_rng(3)
    # keep the symmetric pattern: scale each row and column by the same factors
    d = torch.tensor(1.0 + 0.01 * rng.random(n), device="cuda")
    r = torch.repeat_interleave(torch.arange(n, device="cuda"), rowptr[1:] - rowptr[:-1])
    val2 = val * d[r] * d[col.long()]
    A2 = torch.sparse_csr_tensor(rowptr.long(), col.long(), val2, size=(n, n))
    amg.update_matrix(A2)
    b = torch.tensor(rng.standard_normal(n), device="cuda")
    x32 = amg.vcycle_scaled(b, precision="fp32")
    x64 = amg.vcycle_scaled(b, precision="fp64")
    assert torch.linalg.norm(x32 - x64) <= 1e-4 * torch.linalg.norm(x64)
    levels = amg.levels
    def streamed(lv):
        nnz = lv["A"].values().numel()
        col_bytes = 2 if lv["n"] <= 65536 else 4
        return nnz > 512 * lv["n"] and nnz * (4 + col_bytes) >= 48 * 2**20
    assert any(streamed(lv) for lv in levels if not lv["is_coarsest"])
    A0 = csr_from(levels[0]["A"].crow_indices(), levels[0]["A"].col_indices(), levels[0]["A"].values(), n)
    P0 = levels[0]["P"]
    P0 = sp.csr_matrix((to_np(P0.values()), to_np(P0.col_indices()), to_np(P0.crow_indices())),
                       shape=(n, P0.shape[1]))
    Ac = (P0.T @ A0 @ P0).tocsr()
    A1 = csr_from(levels[1]["A"].crow_indices(), levels[1]["A"].col_indices(), levels[1]["A"].values(),
                  levels[1]["n"])
    assert abs(A1 - Ac).max() <= 1e-10 * abs(Ac).max()


def _laplacian_3d(nx, ny, nz, az=0.1, shift=1e-3):
    def d1(m, a):
        return sp.diags([-a * np.ones(m - 1), 2 * a * np.ones(m), -a * np.ones(m - 1)], [-1, 0, 1])
    ix, iy, iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    A = (sp.kron(sp.kron(d1(nx, 1.0), iy), iz) + sp.kron(sp.kron(ix, d1(ny, 1.0)), iz)
         + sp.kron(sp.kron(ix, iy), d1(nz, az)))
    return (A + shift * sp.identity(nx * ny * nz)).tocsr()


def _host_hierarchy(amg):
    """The oracle's V-cycle over the GPU's exported levels (scipy, float64)."""
    ref = oa.AMG.__new__(oa.AMG)
    ref.levels = []
    for lv in amg.levels:
        n = lv["n"]
        A = csr_from(lv["A"].crow_indices(), lv["A"].col_indices(), lv["A"].values(), n)
        P = None
        if not lv["is_coarsest"]:
            Pt = lv["P"]
            P = sp.csr_matrix((to_np(Pt.values()), to_np(Pt.col_indices()), to_np(Pt.crow_indices())),
                              shape=(n, Pt.shape[1]))
        ref.levels.append(dict(A=A, n=n, P=P, inv_relax=to_np(lv["inv_relax"]), is_coarsest=lv["is_coarsest"]))
    return ref


@pytest.mark.parametrize("far", [False, True])
def test_vcycle_with_16bit_row_relative_columns_vs_host(far):
    """Levels of more than 65,536 rows keep their columns as 16-bit offsets from
    the row when every entry lies within 32K of the diagonal (the 3-D grid
    ordering: 64x64x40, bandwidth 2,560), and as int columns when some entry
    does not (far=True adds symmetric couplings 100,000 columns apart).  The
    fp64 V-cycle equals the oracle's V-cycle over the same exported levels."""
    A = _laplacian_3d(64, 64, 40)
    n = A.shape[0]
    assert n > 65536
    if far:
        i = np.arange(0, n - 100000, 997)
        C = sp.coo_matrix((np.full(i.size, -0.05), (i, i + 100000)), shape=(n, n))
        A = (A + C + C.T + sp.diags(np.asarray(abs(C + C.T).sum(axis=1)).ravel())).tocsr()
    amg = gpu_amg(A, coarsest_size=200, seed=1, mixed_precision=True)
    lv0 = amg.levels[0]
    assert lv0["col_index_bytes"] == (4 if far else 2)
    assert lv0["col_row_relative"] == (not far)
    for lv in amg.levels:
        if lv["n"] <= 65536:
            assert lv["col_index_bytes"] == 2 and not lv["col_row_relative"]
    ref = _host_hierarchy(amg)
    rng = np.random.default_rng(5)
    for _ in range(2):
        bs = rng.standard_normal(n)
        v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision="fp64"))
        v_ref = ref.vcycle(0, np.zeros_like(bs), bs)
        assert np.linalg.norm(v - v_ref) <= 1e-10 * np.linalg.norm(v_ref)
        v32 = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision="fp32"))
        assert np.linalg.norm(v32 - v_ref) <= 1e-4 * np.linalg.norm(v_ref)
    # FGMRES to a true residual checked on the host against the original matrix
    b = rng.standard_normal(n)
    x, st = amg.fgmres(torch.tensor(b, device="cuda"), tol=1e-10, norm="equilibrated", precision="mixed")
    assert st["converged"]
    assert np.linalg.norm(A @ to_np(x) - b) <= 1e-8 * np.linalg.norm(b)


def test_amg_solve_values_cache_and_precision(golden):
    """The drop-in ``amg_solve`` (pressure_amg.py:35-89) by value: the stand-alone
    V-cycles equal the oracle's ``AMGSolver`` on the first recorded matrix and,
    after a cache hit refreshes the hierarchy with ``update_matrix``, on the
    second.  A mixed-precision FGMRES call on the same matrix gets its own
    cached hierarchy (the cache key holds the precision) and reaches the direct
    solution; so does the cache-hit call after it."""
    from impes_b200 import amg as gamg
    from oracle.amg import AMGSolver
    t = golden("two_phase_32x32")
    n = len(t["A0_crow"]) - 1
    mats = [sp.csr_matrix((t["A_val_all"][q], t["A0_col"], t["A0_crow"]), shape=(n, n)) for q in (0, 1)]
    rhs = [t["b_all"][q] for q in (0, 1)]
    gamg._AMG_CACHE.clear()
    ref = AMGSolver(tol=1e-30, max_cycles=5, coarsest_size=50, seed=3)

    def torch_csr(A):
        return torch.sparse_csr_tensor(torch.tensor(A.indptr, dtype=torch.int64),
                                       torch.tensor(A.indices, dtype=torch.int64),
                                       torch.tensor(A.data), size=A.shape)

    for q in (0, 1):
        x_ref = ref(mats[q], rhs[q])
        x = gamg.amg_solve(torch_csr(mats[q]), torch.tensor(rhs[q], device="cuda"), tol=1e-30,
                           max_cycles=5, coarsest_size=50, seed=3)
        assert x.dtype == torch.float64
        assert np.linalg.norm(to_np(x) - x_ref) <= 1e-8 * np.linalg.norm(x_ref), q
        xm = gamg.amg_solve(torch_csr(mats[q]), torch.tensor(rhs[q], device="cuda"), tol=1e-13,
                            max_cycles=300, coarsest_size=50, seed=3, method="fgmres", norm="jacobi",
                            precision="mixed")
        x_direct = spla.spsolve(mats[q].tocsc(), rhs[q])
        assert np.abs(to_np(xm) - x_direct).max() <= 1e-8 * np.abs(x_direct).max(), q
    keys = sorted(k[-2] for k in gamg._AMG_CACHE)
    assert keys == [False, True]
    # a float32 right-hand side comes back as float32 (the reference casts back to b's dtype)
    xf = gamg.amg_solve(torch_csr(mats[1]), torch.tensor(rhs[1], device="cuda").float(), tol=1e-30,
                        max_cycles=5, coarsest_size=50, seed=3)
    assert xf.dtype == torch.float32
    gamg._AMG_CACHE.clear()


@pytest.mark.parametrize("kmax,tf", [(2, 0.0), (4, 0.0), (3, 0.25)])
def test_truncated_hierarchy_matches_oracle(golden, kmax, tf):
    """Interpolation truncation (an option of this library): the same levels,
    P patterns and values as the oracle's restatement of the rule, on a 3-D
    black-oil pressure matrix; the hierarchy is smaller than the reference's."""
    t = golden("black_oil_10x10x4")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = gpu_amg(A, coarsest_size=20, seed=7, p_max_elements=kmax, p_trunc_factor=tf)
    ref = oa.AMG(A, coarsest_size=20, seed=7, p_max_elements=kmax, p_trunc_factor=tf)
    compare_hierarchy(amg, ref)
    full = oa.AMG(A, coarsest_size=20, seed=7)
    assert sum(lv["A"].nnz for lv in ref.levels) < sum(lv["A"].nnz for lv in full.levels)
    for lv in ref.levels:
        if lv["P"] is not None and kmax:
            lens = np.diff(lv["P"].indptr)
            assert lens.max() <= kmax


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["black_oil_10x10x4", "gas_injection_12x12x3", "two_phase_16x16x2"])
def test_truncated_hierarchy_trajectory_matches_reference(golden, name, precision):
    """FGMRES preconditioned by the truncated hierarchy reaches the same pressures
    (1e-8 relative) and saturations (1e-8) as the reference's exact-solve
    trajectory: the preconditioner changes, the solution does not."""
    from gpu_util import cfg_fields, gpu_sim
    g = golden(name)
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-13, norm="jacobi", precision=precision, max_iters=400,
                            restart=40, p_max_elements=2)
    for s in range(g["p"].shape[0]):
        assert sim.run_step(float(g["dt"]))
        assert sim.last_krylov["converged"], sim.last_krylov
        assert np.abs(to_np(fl.pressure) - g["p"][s]).max() <= 1e-8 * np.abs(g["p"][s]).max(), s
        assert np.abs(to_np(fl.s_w) - g["sw"][s]).max() <= 1e-8
        assert np.abs(to_np(fl.s_g) - g["sg"][s]).max() <= 1e-8


@pytest.mark.parametrize("traj,seed,cs", [("two_phase_32x32", 3, 50), ("black_oil_10x10x4", 7, 20)])
def test_chebyshev_vcycle_matches_oracle(golden, traj, seed, cs):
    """The Chebyshev smoother (an option of this library): one V-cycle, a 4-cycle
    stand-alone solve and a solve after update_matrix equal the oracle's
    restatement (1e-9); the fp32 V-cycle stays within fp32 rounding of it."""
    t = golden(traj)
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    A2 = sp.csr_matrix((t["A_val_all"][1], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = gpu_amg(A, coarsest_size=cs, seed=seed, smoother="chebyshev")
    ref = oa.AMG(A, coarsest_size=cs, seed=seed, smoother="chebyshev")
    compare_hierarchy(amg, ref)
    b = t["b0"]
    bs = ref.Dhalf_inv * b
    v_ref = ref.vcycle(0, np.zeros_like(bs), bs)
    v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda")))
    assert np.linalg.norm(v - v_ref) <= 1e-9 * np.linalg.norm(v_ref)
    vf = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision="mixed"))
    assert np.linalg.norm(vf - v_ref) <= 1e-4 * np.linalg.norm(v_ref)
    x_ref, _, _ = ref.solve(b, tol=1e-30, max_iter=4)
    x = to_np(amg.solve(torch.tensor(b, device="cuda"), tol=1e-30, max_iter=4))
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    amg.update_matrix(A2)
    ref.update_matrix(A2)
    b2 = t["b_all"][1]
    x_ref, _, _ = ref.solve(b2, tol=1e-30, max_iter=3)
    x = to_np(amg.solve(torch.tensor(b2, device="cuda"), tol=1e-30, max_iter=3))
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chebyshev_trajectory_matches_reference(golden, precision):
    """FGMRES with Chebyshev-smoothed V-cycles reaches the reference's
    exact-solve trajectory (p 1e-8 relative, S 1e-8) on the black-oil case."""
    from gpu_util import cfg_fields, gpu_sim
    g = golden("black_oil_10x10x4")
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-13, norm="jacobi", precision=precision, max_iters=400,
                            restart=40, smoother="chebyshev")
    for s in range(g["p"].shape[0]):
        assert sim.run_step(float(g["dt"]))
        assert sim.last_krylov["converged"], sim.last_krylov
        assert np.abs(to_np(fl.pressure) - g["p"][s]).max() <= 1e-8 * np.abs(g["p"][s]).max(), s
        assert np.abs(to_np(fl.s_w) - g["sw"][s]).max() <= 1e-8
        assert np.abs(to_np(fl.s_g) - g["sg"][s]).max() <= 1e-8


@pytest.mark.parametrize("traj,seed,cs,light", [("two_phase_32x32", 3, 20, 200),
                                                 ("black_oil_10x10x4", 7, 20, 100),
                                                 ("black_oil_10x10x4", 7, 20, 10 ** 6)])
@pytest.mark.parametrize("smoother", ["l1jacobi", "chebyshev"])
def test_light_sweep_vcycle_matches_oracle(golden, traj, seed, cs, light, smoother):
    """light_sweep_rows (an option of this library): the levels of at most that
    many rows smooth once before and once after their coarse correction.  One
    V-cycle, a 4-cycle stand-alone solve and a solve after update_matrix equal
    the oracle's restatement (1e-9); the fp32 V-cycle stays within fp32
    rounding of it.  The largest threshold makes every level light, level 0
    included."""
    t = golden(traj)
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    A2 = sp.csr_matrix((t["A_val_all"][1], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = gpu_amg(A, coarsest_size=cs, seed=seed, smoother=smoother, light_sweep_rows=light)
    ref = oa.AMG(A, coarsest_size=cs, seed=seed, smoother=smoother, light_sweep_rows=light)
    full = oa.AMG(A, coarsest_size=cs, seed=seed, smoother=smoother)
    compare_hierarchy(amg, ref)
    lv = amg.levels
    assert any(l["n"] <= light and not l["is_coarsest"] for l in lv)
    b = t["b0"]
    bs = ref.Dhalf_inv * b
    v_ref = ref.vcycle(0, np.zeros_like(bs), bs)
    # the option changes the cycle: the light V-cycle is not the reference's
    assert np.linalg.norm(v_ref - full.vcycle(0, np.zeros_like(bs), bs)) > 1e-6 * np.linalg.norm(v_ref)
    v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda")))
    assert np.linalg.norm(v - v_ref) <= 1e-9 * np.linalg.norm(v_ref)
    vf = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision="mixed"))
    assert np.linalg.norm(vf - v_ref) <= 1e-4 * np.linalg.norm(v_ref)
    x_ref, _, _ = ref.solve(b, tol=1e-30, max_iter=4)
    x = to_np(amg.solve(torch.tensor(b, device="cuda"), tol=1e-30, max_iter=4))
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    amg.update_matrix(A2)
    ref.update_matrix(A2)
    b2 = t["b_all"][1]
    x_ref, _, _ = ref.solve(b2, tol=1e-30, max_iter=3)
    x = to_np(amg.solve(torch.tensor(b2, device="cuda"), tol=1e-30, max_iter=3))
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_light_sweep_trajectory_matches_reference(golden, precision):
    """FGMRES preconditioned by light-sweep V-cycles on the capped hierarchy,
    with the whole-step graph, reaches the reference's exact-solve trajectory
    (p 1e-8 relative, S 1e-8) on the gas-injection case."""
    from gpu_util import cfg_fields, gpu_sim
    g = golden("gas_injection_12x12x3")
    cfg, f = cfg_fields(g)
    _, fl, _, sim = gpu_sim(cfg, f, tol=1e-13, norm="jacobi", precision=precision, max_iters=400,
                            restart=40, p_max_elements=2, light_sweep_rows=100)
    for s in range(g["p"].shape[0]):
        assert sim.run_step(float(g["dt"]))
        assert sim.last_krylov["converged"], sim.last_krylov
        assert np.abs(to_np(fl.pressure) - g["p"][s]).max() <= 1e-8 * np.abs(g["p"][s]).max(), s
        assert np.abs(to_np(fl.s_w) - g["sw"][s]).max() <= 1e-8
        assert np.abs(to_np(fl.s_g) - g["sg"][s]).max() <= 1e-8
    graphs, refused = sim.step_graphs()
    assert graphs >= 1 and not refused


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_vcycle_tail_matches_per_level_kernels(monkeypatch, precision):
    """With IMPES_TAIL=1 (read at setup) the levels of at most 4,096 rows run
    as one thread-block-cluster launch per V-cycle (cluster barriers between
    the phases).  Its V-cycle equals the per-level kernels' to rounding: the
    fused kernel sums each row with its own lane count."""
    A = _laplacian_3d(40, 40, 24)
    n = A.shape[0]
    rng = np.random.default_rng(3)
    bs = rng.standard_normal(n)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("IMPES_TAIL", flag)
        amg = gpu_amg(A, coarsest_size=60, seed=2, mixed_precision=True)
        assert amg.levels[0]["n"] > 4096
        v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision=precision))
        x, st = amg.fgmres(torch.tensor(bs, device="cuda"), tol=1e-10, norm="jacobi", precision=precision)
        assert st["converged"], st
        out[flag] = (v, to_np(x), st["iterations"])
        amg.close()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.linalg.norm(out["0"][0] - out["1"][0]) <= tol * np.linalg.norm(out["0"][0])
    assert np.linalg.norm(out["0"][1] - out["1"][1]) <= 1e-8 * np.linalg.norm(out["0"][1])
    assert abs(out["0"][2] - out["1"][2]) <= 1


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sell_and_dia_sweeps_match_csr(monkeypatch, precision):
    """IMPES_SELL=1 (read at setup) puts every level of >= 8,192 rows on its
    SELL-32 copy of A (rows sorted by length inside small windows, 1, 4 or 8
    lanes per row by mean row length); IMPES_DIA=1 puts level 0 of a 7-point
    matrix on its DIA copy (one array per diagonal), with IMPES_DIA_TILE=1 its
    sweeps on grid tiles (two per launch); IMPES_NO_SELL=1 keeps the
    CSR kernels.  The V-cycle and the FGMRES solution agree to rounding: every
    layout adds a row's products lane by lane in the row's order, each with its
    own lanes per row."""
    A = _laplacian_3d(48, 40, 24)
    n = A.shape[0]
    rng = np.random.default_rng(4)
    bs = rng.standard_normal(n)
    out = {}
    slot = 0 if precision == "fp64" else 1
    for mode in ("csr", "sell", "dia", "dia-tile"):
        monkeypatch.setenv("IMPES_NO_SELL", "1" if mode == "csr" else "0")
        monkeypatch.setenv("IMPES_SELL", "1" if mode == "sell" else "0")
        monkeypatch.setenv("IMPES_DIA", "1" if mode.startswith("dia") else "0")
        monkeypatch.setenv("IMPES_DIA_TILE", "1" if mode == "dia-tile" else "0")
        amg = gpu_amg(A, coarsest_size=60, seed=2, mixed_precision=True)
        used = [lv["layout"][slot] for lv in amg.levels if not lv["is_coarsest"]]
        if mode == "csr":
            assert set(used) == {"csr"}, used
        elif mode == "sell":
            assert used[0] == "sell" and used.count("sell") >= 2, used
        else:
            assert used[0] == mode, used
        v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision=precision))
        x, st = amg.fgmres(torch.tensor(bs, device="cuda"), tol=1e-10, norm="jacobi", precision=precision)
        assert st["converged"], st
        out[mode] = (v, to_np(x), st["iterations"])
        amg.close()
    tol = 1e-12 if precision == "fp64" else 1e-5
    for mode in ("sell", "dia", "dia-tile"):
        assert np.linalg.norm(out["csr"][0] - out[mode][0]) <= tol * np.linalg.norm(out[mode][0]), mode
        assert np.linalg.norm(out["csr"][1] - out[mode][1]) <= 1e-8 * np.linalg.norm(out[mode][1]), mode
        assert abs(out["csr"][2] - out[mode][2]) <= 1, mode


@pytest.mark.parametrize("dims", [(45, 37, 19), (64, 48, 3), (24, 10, 40)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_grid_tile_sweeps_match_dia(monkeypatch, dims, precision):
    """With IMPES_DIA_TILE=1, on a grid's 7-point level 0 the two sweeps before
    the residual (with the residual) and the two after the coarse correction
    run as one grid-tile launch each (k_dia_tile: 16 x 10 columns, halos in
    shared memory).  Grids
    that tiles do not divide, a thin and a tall one: the V-cycle, a 4-cycle
    stand-alone solve from a non-zero iterate (one sweep before the tile
    launch) and the FGMRES solution equal the per-pass DIA kernels' (same row
    expression, same order) to the last bits."""
    A = _laplacian_3d(*dims)
    n = A.shape[0]
    rng = np.random.default_rng(7)
    bs = rng.standard_normal(n)
    slot = 0 if precision == "fp64" else 1
    out = {}
    for tile in ("0", "1"):
        monkeypatch.setenv("IMPES_DIA", "1")
        monkeypatch.setenv("IMPES_DIA_TILE", tile)
        amg = gpu_amg(A, coarsest_size=60, seed=2, mixed_precision=True)
        assert amg.levels[0]["layout"][slot] == ("dia-tile" if tile == "1" else "dia")
        v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision=precision))
        xs = to_np(amg.solve(torch.tensor(bs, device="cuda"), tol=1e-30, max_iter=4)) if precision == "fp64" else None
        x, st = amg.fgmres(torch.tensor(bs, device="cuda"), tol=1e-10, norm="jacobi", precision=precision)
        assert st["converged"], st
        out[tile] = (v, xs, to_np(x), st["iterations"])
        amg.close()
    (v0, s0, x0, i0), (v1, s1, x1, i1) = out["0"], out["1"]
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert np.linalg.norm(v1 - v0) <= tol * np.linalg.norm(v0)
    if s0 is not None:
        assert np.linalg.norm(s1 - s0) <= 1e-13 * np.linalg.norm(s0)
    assert np.linalg.norm(x1 - x0) <= 1e-8 * np.linalg.norm(x0)
    assert abs(i1 - i0) <= 1


def test_tuner_choices_persist_across_processes(tmp_path, monkeypatch):
    """IMPES_TUNE_CACHE=<file>: the lanes-per-row and layout choices of a
    hierarchy are written to the file, and another process that loads it
    launches the same kernels for a hierarchy of the same shape, whatever its
    own timings would say."""
    import json
    import subprocess
    import sys
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("IMPES_TUNE_CACHE", str(cache))
    A = _laplacian_3d(40, 40, 24)
    amg = gpu_amg(A, coarsest_size=60, seed=2, mixed_precision=True)
    mine = [(lv["n"], lv["lanes"], lv["layout"]) for lv in amg.levels]
    amg.close()
    lines = cache.read_text().split("\n")
    rows = [list(map(int, ln.split())) for ln in lines if ln.strip()]
    assert rows and all(len(r) == 5 for r in rows)
    code = ("import sys, json; sys.path[:0] = %r\n"
            "from test_gpu_amg import _laplacian_3d, gpu_amg\n"
            "a = gpu_amg(_laplacian_3d(40, 40, 24), coarsest_size=60, seed=2, mixed_precision=True)\n"
            "print(json.dumps([(lv['n'], lv['lanes'], lv['layout']) for lv in a.levels]))\n") % (sys.path,)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                         cwd=str(tmp_path), env=dict(__import__("os").environ))
    assert out.returncode == 0, out.stderr[-2000:]
    theirs = json.loads(out.stdout.strip().splitlines()[-1])
    assert [(n, tuple(ln), tuple(l)) for n, ln, l in theirs] == mine


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_shared_memory_tail_matches_per_level_kernels(monkeypatch, precision):
    """With IMPES_STAIL=1 (read at setup) the fp32 V-cycle of the smallest
    levels runs as one 1024-thread CTA with their matrices, transfers and
    vectors staged in shared memory.  Its V-cycle equals the per-level
    kernels' to rounding (it sums each row with four lanes); the fp64 V-cycle
    never uses it."""
    A = _laplacian_3d(40, 40, 24)
    n = A.shape[0]
    rng = np.random.default_rng(5)
    bs = rng.standard_normal(n)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("IMPES_STAIL", flag)
        amg = gpu_amg(A, coarsest_size=60, seed=2, mixed_precision=True)
        tail = [lv["fused_tail"] for lv in amg.levels]
        if flag == "1":
            assert "shared" in tail and tail[0] is None, tail
        else:
            assert "shared" not in tail, tail
        v = to_np(amg.vcycle_scaled(torch.tensor(bs, device="cuda"), precision=precision))
        x, st = amg.fgmres(torch.tensor(bs, device="cuda"), tol=1e-10, norm="jacobi", precision=precision)
        assert st["converged"], st
        out[flag] = (v, to_np(x), st["iterations"])
        amg.close()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.linalg.norm(out["0"][0] - out["1"][0]) <= tol * np.linalg.norm(out["0"][0])
    assert np.linalg.norm(out["0"][1] - out["1"][1]) <= 1e-8 * np.linalg.norm(out["0"][1])
    assert abs(out["0"][2] - out["1"][2]) <= 1
