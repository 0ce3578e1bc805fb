"""Classical AMG pressure solver on the B200, behind the reference's Python API.

Mirrors researchim-ai/oil-simulator-py ``src/solver/classical_amg.py``
(``ClassicalAMG`` :694-1392, ``_apply_reference_fix`` :660-686) and
``src/solver/pressure_amg.py`` (``amg_solve`` :35-89, ``amg_preconditioner``
:92-160, the module-level ``_AMG_CACHE`` :8).  All arithmetic runs in
``libimpes_b200.so``; matrices and vectors live on the current CUDA device.

Differences from the reference, by design:

* the C/F tie-break is a deterministic stream (``seed``) instead of
  ``torch.rand``, so hierarchies are reproducible and comparable;
* ``fgmres()`` / ``amg_solve(method="fgmres")`` add a flexible GMRES with one
  V-cycle per iteration (fp64 or fp32 V-cycle), stopping in the reference's
  equilibrated norm or in the Jacobi-scaled norm ``||D^-1 r|| / ||D^-1 b||``;
* CPU execution is not offered: a CPU ``device`` raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Dict, Optional, Tuple

import torch

from . import _lib
from ._lib import check, lib, ptr

_NORMS = {"equilibrated": _lib.NORM_EQUILIBRATED, "jacobi": _lib.NORM_JACOBI}
_PRECISION = {"fp64": 0, "float64": 0, "mixed": 1, "fp32": 1}
_SMOOTHERS = {"l1jacobi": 0, "chebyshev": 1}


def _cuda_device(device=None) -> torch.device:
    if device in (None, "auto"):
        dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
    else:
        dev = torch.device(device)
    if dev is None or dev.type != "cuda":
        raise RuntimeError("the B200 AMG runs on CUDA only; no CPU path is provided")
    return dev


def to_csr32(A, device) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, Tuple[int, int]]:
    """(rowptr int32, col int32, values float64, shape) on ``device`` from a torch
    sparse COO/CSR tensor, a dense tensor or a scipy sparse matrix
    (``_to_csr_double``, pressure_amg.py:11-32)."""
    if isinstance(A, tuple) and len(A) == 4:
        return A
    if not isinstance(A, torch.Tensor) and hasattr(A, "tocsr"):
        # scipy sparse, any format: a private CSR copy with duplicates summed and
        # columns sorted (the caller's matrix is left as it was)
        A = A.tocsr(copy=True)
        A.sum_duplicates()
        return (torch.as_tensor(A.indptr, dtype=torch.int32, device=device),
                torch.as_tensor(A.indices, dtype=torch.int32, device=device),
                torch.as_tensor(A.data, dtype=torch.float64, device=device), tuple(A.shape))
    if A.layout == torch.sparse_coo:
        A = A.coalesce().to_sparse_csr()
    elif A.layout != torch.sparse_csr:
        A = A.to_sparse().coalesce().to_sparse_csr()
    return (A.crow_indices().to(device=device, dtype=torch.int32).contiguous(),
            A.col_indices().to(device=device, dtype=torch.int32).contiguous(),
            A.values().to(device=device, dtype=torch.float64).contiguous(), tuple(A.shape))


def _apply_reference_fix(A_csr: torch.Tensor, anchor_idx: int, anchor_value: float = 0.0) -> torch.Tensor:
    """Pin one DOF: drop its row/column, set the diagonal to 1 (classical_amg.py:660-686)."""
    A_coo = A_csr.to_sparse_coo().coalesce()
    row, col = A_coo.indices()
    val = A_coo.values().clone()
    keep = ~((row == anchor_idx) | (col == anchor_idx)) | ((row == anchor_idx) & (col == anchor_idx))
    row, col, val = row[keep], col[keep], val[keep]
    dm = (row == anchor_idx) & (col == anchor_idx)
    if bool(dm.any()):
        val[dm] = 1.0
    else:
        row = torch.cat([row, torch.tensor([anchor_idx], device=row.device)])
        col = torch.cat([col, torch.tensor([anchor_idx], device=col.device)])
        val = torch.cat([val, torch.tensor([1.0], dtype=val.dtype, device=val.device)])
    return torch.sparse_coo_tensor(torch.stack([row, col]), val, A_csr.size(),
                                   device=A_csr.device, dtype=A_csr.dtype).coalesce().to_sparse_csr()


class ClassicalAMG:
    """Ruge--Stueben AMG hierarchy (``ClassicalAMG``, classical_amg.py:694-1392).

    ``seed`` selects the C/F tie-break stream; ``mixed_precision`` keeps an fp32
    copy of every level for the fp32 V-cycle of the mixed path.
    ``p_max_elements`` / ``p_trunc_factor`` truncate the interpolation (an option
    the reference does not have; the defaults keep its interpolation): each F
    row of P keeps at most ``p_max_elements`` entries (0: no cap) and drops those
    below ``p_trunc_factor`` times its largest, rescaled to the old row sum.
    ``smoother`` is "l1jacobi" (the reference's) or "chebyshev" (the Chebyshev
    iteration for diag(l1 weights) A on [``cheb_lower`` * lmax, lmax], lmax its
    Gershgorin bound; also not in the reference).  ``light_sweep_rows``: levels
    of at most that many rows smooth once before and once after their coarse
    correction instead of three and two times (0, the default: the reference's
    V-cycle on every level).
    """

    def __init__(self, A_csr_np, theta: float = 0.25, max_levels: int = 10, coarsest_size: int = 100,
                 anchor_idx: int | None = None, nullspace_dim: int = 3, nullspace_blend: float = 0.6,
                 nullspace_reg: float = 1e-6, *, seed: int = 0, mixed_precision: bool = True,
                 device=None, p_max_elements: int = 0, p_trunc_factor: float = 0.0,
                 smoother: str = "l1jacobi", cheb_lower: float = 0.3, light_sweep_rows: int = 0):
        if anchor_idx is not None:
            raise ValueError("anchor_idx is not supported; pin the matrix with _apply_reference_fix first")
        self.theta, self.max_levels, self.coarsest_size = float(theta), int(max_levels), int(coarsest_size)
        self.anchor_idx = None
        self.nullspace_dim = max(0, int(nullspace_dim))
        self.nullspace_blend = float(max(0.0, min(1.0, nullspace_blend)))
        self.nullspace_reg = float(max(1e-10, nullspace_reg))
        self.apply_tol = 5e-2           # classical_amg.py:724
        self.apply_max_cycles = 8       # classical_amg.py:725
        self.equilibration_threshold = 1e-6
        self.device = _cuda_device(device)
        self.seed = int(seed)
        self.mixed_precision = bool(mixed_precision)
        self.p_max_elements, self.p_trunc_factor = int(p_max_elements), float(p_trunc_factor)
        if smoother not in _SMOOTHERS:
            raise ValueError(f"unknown smoother {smoother!r}")
        self.smoother, self.cheb_lower = smoother, float(cheb_lower)
        self.light_sweep_rows = int(light_sweep_rows)
        prm = _lib.AmgParams(self.theta, self.max_levels, self.coarsest_size, self.nullspace_dim,
                             self.nullspace_blend, self.nullspace_reg, self.equilibration_threshold,
                             self.seed & 0xFFFFFFFF, 1 if self.mixed_precision else 0,
                             self.p_max_elements, self.p_trunc_factor, _SMOOTHERS[smoother],
                             self.cheb_lower, self.light_sweep_rows)
        h = C.c_void_p()
        check(lib.impes_amg_create(C.byref(h), C.byref(prm)), "impes_amg_create")
        self._h = h
        self._levels_cache = None
        self.last_stats: Dict[str, Any] = {}
        rowptr, col, val, shape = to_csr32(A_csr_np, self.device)
        if shape[0] != shape[1]:
            raise ValueError("matrix must be square")
        self.n = shape[0]
        self._pattern = (rowptr, col)
        with torch.cuda.device(self.device):
            check(lib.impes_amg_setup(self._h, self.n, int(col.numel()), ptr(rowptr), ptr(col), ptr(val),
                                      _lib.stream_of(self.device)), "impes_amg_setup")

    # ------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, "_h", None):
            lib.impes_amg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -------------------------------------------------------------- updates
    def update_matrix(self, A_csr_np) -> None:
        """New values on the same pattern (``update_matrix``, classical_amg.py:1308-1392)."""
        rowptr, col, val, shape = to_csr32(A_csr_np, self.device)
        if shape[0] != self.n:
            raise ValueError(f"AMG hierarchy built for n={self.n}, got n={shape[0]}")
        if (col.numel() != self._pattern[1].numel() or not torch.equal(col, self._pattern[1])
                or not torch.equal(rowptr, self._pattern[0])):
            raise ValueError("update_matrix needs the sparsity pattern the hierarchy was built on")
        self.update_values(val)

    def update_values(self, val: torch.Tensor) -> None:
        with torch.cuda.device(self.device):
            check(lib.impes_amg_update(self._h, ptr(val), _lib.stream_of(self.device)), "impes_amg_update")
        self._levels_cache = None

    # -------------------------------------------------------------- solving
    def _vec(self, b):
        return b.to(self.device, dtype=torch.float64).contiguous().reshape(-1)

    def solve(self, b, x0: Optional[torch.Tensor] = None, tol: float = 1e-6, max_iter: int = 10,
              norm: str = "equilibrated") -> torch.Tensor:
        """Stand-alone V-cycles (``solve``, classical_amg.py:1108-1155); ``norm="jacobi"``
        stops on ||D^-1 r|| / ||D^-1 b|| instead of the reference's equilibrated norm."""
        if x0 is not None:
            raise ValueError("x0 is not supported by the V-cycle solve; use fgmres(use_x0=...)")
        bb = self._vec(b)
        x = torch.empty_like(bb)
        cyc, rel = C.c_int(0), C.c_double(0.0)
        with torch.cuda.device(self.device):
            check(lib.impes_amg_solve_vcycles(self._h, ptr(bb), ptr(x), float(tol), int(max_iter),
                                              C.byref(cyc), C.byref(rel), _NORMS[norm],
                                              _lib.stream_of(self.device)),
                  "impes_amg_solve_vcycles")
        self.last_stats = {"cycles": cyc.value, "rel_res": rel.value}
        return x

    def apply(self, b, cycles: int = 1, pre_smooth: int = 3, post_smooth: int = 2) -> torch.Tensor:
        """Incomplete solve (``apply``, classical_amg.py:1157-1180)."""
        if pre_smooth != 3 or post_smooth != 2:
            raise ValueError("the V-cycle uses 3 pre- and 2 post-smoothing sweeps")
        bb = self._vec(b)
        x = torch.empty_like(bb)
        with torch.cuda.device(self.device):
            check(lib.impes_amg_apply(self._h, ptr(bb), ptr(x), int(cycles), float(self.apply_tol),
                                      int(self.apply_max_cycles), _lib.stream_of(self.device)),
                  "impes_amg_apply")
        return x

    def vcycle_scaled(self, b_scaled, precision: str = "fp64") -> torch.Tensor:
        """One V-cycle on the equilibrated system from x = 0 (``_v_cycle(0, 0, b_s)``)."""
        bb = self._vec(b_scaled)
        x = torch.empty_like(bb)
        with torch.cuda.device(self.device):
            check(lib.impes_amg_vcycle_scaled(self._h, ptr(bb), ptr(x), _PRECISION[precision],
                                              _lib.stream_of(self.device)), "impes_amg_vcycle_scaled")
        return x

    def fgmres(self, b, tol: float = 1e-6, restart: int = 60, max_iters: int = 300,
               norm: str = "jacobi", precision: str = "fp64", x0: Optional[torch.Tensor] = None):
        """FGMRES with one V-cycle per iteration.  Returns (x, stats dict)."""
        bb = self._vec(b)
        x = torch.zeros_like(bb) if x0 is None else self._vec(x0).clone()
        kp = _lib.KrylovParams(float(tol), int(restart), int(max_iters), _NORMS[norm],
                               _PRECISION[precision], 0 if x0 is None else 1)
        st = _lib.KrylovStats()
        with torch.cuda.device(self.device):
            check(lib.impes_amg_fgmres(self._h, ptr(bb), ptr(x), C.byref(kp), C.byref(st),
                                       _lib.stream_of(self.device)), "impes_amg_fgmres")
        self.last_stats = {"iterations": st.iterations, "restarts": st.restarts,
                           "converged": bool(st.converged), "rel_res": st.rel_res,
                           "true_rel_res": st.true_rel_res}
        return x, dict(self.last_stats)

    # --------------------------------------------------------- introspection
    @property
    def Dhalf_inv(self) -> Optional[torch.Tensor]:
        en = C.c_int(0)
        out = torch.empty(self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(lib.impes_amg_equilibration(self._h, ptr(out), C.byref(en), _lib.stream_of(self.device)),
                  "impes_amg_equilibration")
        return out if en.value else None

    @property
    def use_equilibration(self) -> bool:
        return self.Dhalf_inv is not None

    @property
    def levels(self):
        """List of level dicts with keys A, n, P, inv_relax, diag, is_coarsest, and the
        column storage of the level's sweeps: col_index_bytes (2 or 4) and
        col_row_relative (16-bit offsets from the row)."""
        if self._levels_cache is not None:
            return self._levels_cache
        nl = C.c_int(0)
        check(lib.impes_amg_num_levels(self._h, C.byref(nl)))
        out = []
        dev = self.device
        for l in range(nl.value):
            info = _lib.LevelDesc()
            check(lib.impes_amg_level_info(self._h, l, C.byref(info)))
            ar = torch.empty(info.n + 1, dtype=torch.int32, device=dev)
            ac = torch.empty(max(info.nnz, 1), dtype=torch.int32, device=dev)
            av = torch.empty(max(info.nnz, 1), dtype=torch.float64, device=dev)
            ir = torch.empty(info.n, dtype=torch.float64, device=dev)
            pr = pc = pv = None
            if not info.is_coarsest:
                pr = torch.empty(info.n + 1, dtype=torch.int32, device=dev)
                pc = torch.empty(max(info.p_nnz, 1), dtype=torch.int32, device=dev)
                pv = torch.empty(max(info.p_nnz, 1), dtype=torch.float64, device=dev)
            with torch.cuda.device(dev):
                check(lib.impes_amg_level_export(self._h, l, ptr(ar), ptr(ac), ptr(av), ptr(ir), ptr(pr),
                                                 ptr(pc), ptr(pv), _lib.stream_of(dev)))
            A = torch.sparse_csr_tensor(ar.long(), ac[:info.nnz].long(), av[:info.nnz], size=(info.n, info.n))
            P = None
            if not info.is_coarsest:
                P = torch.sparse_csr_tensor(pr.long(), pc[:info.p_nnz].long(), pv[:info.p_nnz],
                                            size=(info.n, info.p_cols))
            diag = A.to_sparse_coo().coalesce()
            idx = diag.indices()
            dmask = idx[0] == idx[1]
            d = torch.zeros(info.n, dtype=torch.float64, device=dev)
            d[idx[0][dmask]] = diag.values()[dmask]
            out.append({"A": A, "n": info.n, "P": P, "inv_relax": ir, "diag": d.abs(),
                        "is_coarsest": bool(info.is_coarsest),
                        "col_index_bytes": info.col_index_bytes,
                        "col_row_relative": bool(info.col_row_relative),
                        "lanes": tuple(info.lanes),
                        "fused_tail": {0: None, 1: "shared", 2: "cluster"}[info.fused_tail],
                        "layout": tuple({0: "csr", 1: "sell", 2: "dia", 3: "dia-tile"}[v] for v in info.layout)})
        self._levels_cache = out
        return out

    def _matvec(self, lvl: int, x: torch.Tensor) -> torch.Tensor:
        A = self.levels[lvl]["A"]
        return torch.sparse.mm(A, x.unsqueeze(1)).squeeze(1)


# ------------------------------------------------------------------ module API
_AMG_CACHE: Dict[Tuple[Any, ...], ClassicalAMG] = {}


def amg_solve(A, b: torch.Tensor, *, tol: float = 1e-6, max_cycles: int = 20, theta: float = 0.25,
              max_levels: int = 10, coarsest_size: int = 200, device: Optional[str] = "auto",
              enable_equilibration: Optional[bool] = None, method: str = "vcycle",
              norm: str = "equilibrated", precision: str = "fp64", restart: int = 60,
              max_iters: Optional[int] = None, seed: int = 0) -> torch.Tensor:
    """Solve A x = b (``amg_solve``, pressure_amg.py:35-89).

    ``method="vcycle"`` (default) keeps the reference's stand-alone V-cycles and
    stopping rule; ``method="fgmres"`` runs FGMRES to ``tol`` in ``norm`` with at
    most ``max_iters`` (default ``max_cycles``) V-cycles.  The hierarchy is cached
    per (size, theta, max_levels, coarsest_size, device) as the reference's
    ``_AMG_CACHE`` is, plus the two settings the reference does not have: whether
    the hierarchy keeps fp32 levels (``precision`` other than "fp64") and the
    tie-break ``seed``.  A hit on the same pattern (row pointers and columns)
    is refreshed with ``update_matrix``; a different pattern rebuilds.  Returns x
    on b's device and dtype.
    """
    if precision not in _PRECISION:
        raise ValueError(f"unknown precision {precision!r}")
    dev = _cuda_device(device)
    rowptr, col, val, shape = to_csr32(A, dev)
    mixed = _PRECISION[precision] == 1
    key = (torch.Size(shape), float(theta), int(max_levels), int(coarsest_size), str(dev), mixed,
           int(seed))
    amg = _AMG_CACHE.get(key)
    same_pattern = (amg is not None and rowptr.numel() == amg._pattern[0].numel()
                    and col.numel() == amg._pattern[1].numel()
                    and torch.equal(rowptr, amg._pattern[0]) and torch.equal(col, amg._pattern[1]))
    if amg is None or not same_pattern:
        amg = ClassicalAMG((rowptr, col, val, shape), theta=theta, max_levels=max_levels,
                           coarsest_size=coarsest_size, seed=seed, device=dev, mixed_precision=mixed)
        _AMG_CACHE[key] = amg
    else:
        amg.update_values(val)
    if method == "vcycle":
        x = amg.solve(b, tol=tol, max_iter=max_cycles)
    elif method == "fgmres":
        x, _ = amg.fgmres(b, tol=tol, restart=restart, max_iters=max_iters or max_cycles, norm=norm,
                          precision=precision)
    else:
        raise ValueError(f"unknown method {method!r}")
    return x.to(b.device, dtype=b.dtype)


def amg_preconditioner(A, *, theta: float = 0.25, max_levels: int = 10, coarsest_size: int = 200,
                       device: Optional[str] = "auto", seed: int = 0) -> Dict[str, Any]:
    """Right preconditioner M(r) ~ A^-1 by one V-cycle (``amg_preconditioner``,
    pressure_amg.py:92-160): tries theta candidates until ``apply(v, 2)`` reaches
    a 5e-2 relative residual on a constant, a random and a ramp vector."""
    dev = _cuda_device(device)
    csr = to_csr32(A, dev)
    A_t = torch.sparse_csr_tensor(csr[0].long(), csr[1].long(), csr[2], size=csr[3])
    n = csr[3][0]
    gen = torch.Generator(device=dev).manual_seed(seed)

    def quality(amg):
        tests = [torch.ones(n, dtype=torch.float64, device=dev),
                 torch.randn(n, dtype=torch.float64, device=dev, generator=gen),
                 torch.linspace(0, 1, n, dtype=torch.float64, device=dev)]
        rels = []
        for v in tests:
            v = v / (v.norm() + 1e-30)
            z = amg.apply(v, cycles=2)
            rels.append(float(((torch.sparse.mm(A_t, z.unsqueeze(1)).squeeze(1) - v).norm()
                               / (v.norm() + 1e-30))))
        return max(rels)

    cands = [theta] + ([0.2] if theta > 0.2 else []) + [0.15, 0.1]
    chosen, best, best_amg = None, float("inf"), None
    for th in cands:
        amg = ClassicalAMG(csr, theta=th, max_levels=max_levels, coarsest_size=coarsest_size,
                           seed=seed, device=dev)
        sc = quality(amg)
        if sc < best:
            best, best_amg = sc, amg
        if sc <= 0.05:
            chosen = amg
            break
    if chosen is None:
        raise RuntimeError(f"AMG preconditioner quality too low (best score={best:.3e})")

    def _apply(r: torch.Tensor) -> torch.Tensor:
        return chosen.apply(r, cycles=1).to(r.device, dtype=r.dtype)

    return {"apply": _apply, "device": chosen.device}
