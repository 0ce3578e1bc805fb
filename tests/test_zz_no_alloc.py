"""impes_amg_solve_vcycles_noalloc against impes_amg_solve_vcycles, through the C ABI.

The no-alloc entry point keeps its work vectors in a static device array; its
results must equal the allocating solve's on consecutive calls (the array is
reused, so a second call must not see the first call's leftovers)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

pytestmark = pytest.mark.gpu

MAX_ROWS = 262144


def _laplacian_3d(nx, ny, nz, az=0.1):
    def d1(m, a):
        return sp.diags([-a * np.ones(m - 1), 2 * a * np.ones(m), -a * np.ones(m - 1)], [-1, 0, 1])
    ix, iy, iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    A = (sp.kron(sp.kron(d1(nx, 1.0), iy), iz) + sp.kron(sp.kron(ix, d1(ny, 1.0)), iz)
         + sp.kron(sp.kron(ix, iy), d1(nz, az)))
    return (A + 1e-3 * sp.identity(nx * ny * nz)).tocsr()


def _solve(entry, amg, b, tol, cycles, norm):
    from impes_b200 import _lib
    x = torch.full_like(b, 7.0)
    cyc, rel = C.c_int(), C.c_double()
    status = getattr(_lib.lib, entry)(amg.handle, _lib.ptr(b), _lib.ptr(x), float(tol), int(cycles),
                                      C.byref(cyc), C.byref(rel), int(norm), _lib.stream_of(b.device))
    torch.cuda.synchronize()
    return status, x, cyc.value, rel.value


@pytest.mark.parametrize("norm", [0, 1])
@pytest.mark.parametrize("shape", ["golden_32x32", "laplace_3d"])
def test_noalloc_matches_allocating_solve(golden, shape, norm):
    from impes_b200.amg import ClassicalAMG
    if shape == "golden_32x32":
        t = golden("two_phase_32x32")
        n = len(t["A0_crow"]) - 1
        A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    else:
        A = _laplacian_3d(40, 40, 24)
        n = A.shape[0]
    amg = ClassicalAMG(A, coarsest_size=50, seed=3)
    rng = np.random.default_rng(11)
    for call in range(2):
        b = torch.tensor(rng.standard_normal(n), device="cuda", dtype=torch.float64)
        s0, x0, c0, r0 = _solve("impes_amg_solve_vcycles", amg, b, 1e-8, 40, norm)
        s1, x1, c1, r1 = _solve("impes_amg_solve_vcycles_noalloc", amg, b, 1e-8, 40, norm)
        assert s0 == 0 and s1 == 0, call
        assert c1 == c0 and abs(r1 - r0) <= 1e-12 * max(r0, 1e-300), (call, c0, c1, r0, r1)
        assert torch.linalg.norm(x1 - x0) <= 1e-12 * torch.linalg.norm(x0), call


def test_noalloc_rejects_more_rows_than_its_work_space():
    from impes_b200 import _lib
    from impes_b200.amg import ClassicalAMG
    A = _laplacian_3d(66, 66, 62)         # 270072 rows > 262144
    assert A.shape[0] > MAX_ROWS
    amg = ClassicalAMG(A, coarsest_size=200, seed=0)
    b = torch.ones(A.shape[0], device="cuda", dtype=torch.float64)
    status, x, _, _ = _solve("impes_amg_solve_vcycles_noalloc", amg, b, 1e-6, 3, 0)
    assert status == _lib.ERR_ARG
    assert b"262144" in _lib.lib.impes_last_error()
    assert bool(torch.all(x == 7.0))
    # the handle stays usable
    s, _, _, _ = _solve("impes_amg_solve_vcycles", amg, b, 1e-6, 3, 0)
    assert s == 0


def test_noalloc_after_fp32_update_of_a_mixed_hierarchy(golden):
    """A mixed-precision hierarchy refreshed by update_matrix holds only its fp32
    Galerkin chain; the fp64 levels are rebuilt on the next fp64 solve.  The
    no-alloc solve runs first after each update, so it is the call that rebuilds
    them (into the buffers made at setup), and must still equal the allocating
    solve, on two consecutive updates."""
    from impes_b200.amg import ClassicalAMG
    t = golden("two_phase_32x32")
    n = len(t["A0_crow"]) - 1
    A = sp.csr_matrix((t["A0_val"], t["A0_col"], t["A0_crow"]), shape=(n, n))
    amg = ClassicalAMG(A, coarsest_size=50, seed=3, mixed_precision=True)
    rng = np.random.default_rng(5)
    for call, q in enumerate((1, 2)):
        val = torch.tensor(t["A_val_all"][q], device="cuda", dtype=torch.float64)
        amg.update_values(val)
        b = torch.tensor(t["b_all"][q], device="cuda", dtype=torch.float64)
        b = b + 1e-3 * b.abs().max() * torch.tensor(rng.standard_normal(n), device="cuda")
        s1, x1, c1, r1 = _solve("impes_amg_solve_vcycles_noalloc", amg, b, 1e-9, 30, 1)
        s0, x0, c0, r0 = _solve("impes_amg_solve_vcycles", amg, b, 1e-9, 30, 1)
        assert s0 == 0 and s1 == 0, call
        assert c1 == c0 and abs(r1 - r0) <= 1e-12 * max(r0, 1e-300), (call, c0, c1, r0, r1)
        assert torch.linalg.norm(x1 - x0) <= 1e-12 * torch.linalg.norm(x0), call
