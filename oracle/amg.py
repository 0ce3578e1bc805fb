"""Float64 CPU restatement of the reference's classical Ruge--Stueben AMG (checker only).

Follows researchim-ai/oil-simulator-py ``src/solver/classical_amg.py``:

* ``find_strong_connections``      :34-82
* ``classical_coarsening``         :85-146 (the ``torch.rand`` tie-break at :125 is an
  input here, see ``tiebreak``)
* ``build_prolongation_rs_full``   :149-427 (orphan promotion, direct + F-F
  weights, weak correction, clamp, row normalisation with injection fallback,
  energy blend through ``solve_energy_weights`` :1469-1501)
* ``rap_torch``                    :653-657 (Galerkin P^T A P)
* ``ClassicalAMG.__init__``        :699-938 (equilibration :763-788, level loop)
* ``_v_cycle`` / ``solve`` / ``apply`` :1037-1180, ``update_matrix`` :1308-1392
* ``generate_nullspace`` / ``orthonormalize_columns`` :1395-1466

and ``src/solver/pressure_amg.py:35-89`` (``amg_solve`` with its hierarchy cache).

Matrices are scipy CSR with sorted indices, float64.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

_M64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea & Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def tiebreak(seed: int, level: int, n: int) -> np.ndarray:
    """Uniform [0,1) float64 tie-break for C/F selection at ``level``.

    The reference draws ``torch.rand(n)`` (classical_amg.py:125); the build takes
    the vector as an input so that CPU and GPU hierarchies can be compared.  Key
    = seed<<40 | level<<32 | i, value = top 53 bits of splitmix64(key) / 2^53.
    """
    i = np.arange(n, dtype=np.uint64)
    key = (np.uint64((seed & 0xFFFFFF) << 40) | np.uint64((level & 0xFF) << 32)) | i
    return (splitmix64(key) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _row_idx(A):
    return np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))


def extract_diag(A):
    """``ClassicalAMG._extract_diag`` (classical_amg.py:940-955)."""
    r = _row_idx(A)
    d = np.zeros(A.shape[0])
    m = r == A.indices
    d[r[m]] = A.data[m]
    return d


def strength(A, theta):
    """``find_strong_connections`` (classical_amg.py:34-82): bool per stored entry."""
    r = _row_idx(A)
    col, vals = A.indices, A.data
    n = A.shape[0]
    diag = np.zeros(n)
    dm = r == col
    diag[r[dm]] = np.abs(vals[dm])
    svals = vals / (np.abs(diag[r]) + 1e-30)
    cand = (col != r) & (svals < 0)
    neg_abs = np.where(cand, -svals, 0.0)
    mx = np.zeros(n)
    np.maximum.at(mx, r, neg_abs)
    return cand & (neg_abs >= theta * mx[r])


def transpose_positions(A):
    """Position of entry (j, i) for every stored (i, j); -1 where absent."""
    r = _row_idx(A)
    n = A.shape[0]
    key = r.astype(np.int64) * n + A.indices
    tkey = A.indices.astype(np.int64) * n + r
    order = np.argsort(key)
    pos = np.searchsorted(key[order], tkey)
    pos = np.clip(pos, 0, len(key) - 1)
    hit = key[order][pos] == tkey
    return np.where(hit, order[pos], -1)


def coarsen(A, theta, w):
    """``classical_coarsening`` (classical_amg.py:85-146) with tie-break ``w``.

    Returns cf (0 = C, 1 = F) and the number of C points.
    """
    n = A.shape[0]
    r = _row_idx(A)
    s = strength(A, theta)
    i, j = r[s], A.indices[s]
    e0, e1 = np.minimum(i, j), np.maximum(i, j)
    ed = np.unique(e0.astype(np.int64) * n + e1)
    ii, jj = ed // n, ed % n
    deg = np.zeros(n)
    np.add.at(deg, ii, 1.0)
    np.add.at(deg, jj, 1.0)
    score = deg + 1e-3 * w
    # Two scatter_reduce_(amax, include_self=False) passes (:131-132): the second
    # pass REPLACES the value of every node it touches, so a node's neighbour max
    # is taken over its lower-index strong neighbours when it has any, else over
    # its higher-index ones, else it stays 0.
    up = np.full(n, -np.inf)
    np.maximum.at(up, ii, score[jj])
    lo = np.full(n, -np.inf)
    np.maximum.at(lo, jj, score[ii])
    has_lo = np.zeros(n, dtype=bool); has_lo[jj] = True
    has_up = np.zeros(n, dtype=bool); has_up[ii] = True
    nm = np.where(has_lo, lo, np.where(has_up, up, 0.0))
    C = score > nm
    cf = np.where(C, 0, 1).astype(np.int8)
    hasC = np.zeros(n, dtype=np.int64)
    np.add.at(hasC, ii, C[jj].astype(np.int64))
    np.add.at(hasC, jj, C[ii].astype(np.int64))
    cf[(cf == 1) & (hasC == 0)] = 0
    return cf, int((cf == 0).sum())


def orthonormalize(B):
    """``orthonormalize_columns`` (classical_amg.py:1395-1407), classical Gram-Schmidt."""
    cols = []
    for c in range(B.shape[1]):
        v = B[:, c].copy()
        for q in cols:
            v = v - np.dot(v, q) * q
        nv = np.linalg.norm(v)
        if nv > 1e-10:
            cols.append(v / nv)
    if not cols:
        v = np.ones(B.shape[0])
        cols.append(v / (np.linalg.norm(v) + 1e-30))
    return np.stack(cols, axis=1)


def nullspace(n, dim=3):
    """``generate_nullspace`` (classical_amg.py:1426-1466) for ``dim <= 3``.

    With dim <= 3 the basis is the constant, a centred index ramp and a centred
    index-squared ramp (the random smoothed vectors at :1450-1462 only run for
    dim > 3).
    """
    if dim <= 0:
        return None
    basis = [np.ones(n) / (np.linalg.norm(np.ones(n)) + 1e-30)]
    coords = np.linspace(0.0, 1.0, n)
    centered = coords - coords.mean()
    if np.linalg.norm(centered) > 1e-8 and len(basis) < dim:
        basis.append(centered / np.linalg.norm(centered))
    poly = coords ** 2 - (coords ** 2).mean()
    if np.linalg.norm(poly) > 1e-8 and len(basis) < dim:
        poly = poly - sum(np.dot(poly, b) * b for b in basis)
        if np.linalg.norm(poly) > 1e-8:
            basis.append(poly / np.linalg.norm(poly))
    if dim > 3:
        raise NotImplementedError("nullspace_dim > 3 is not restated")
    return orthonormalize(np.stack(basis, axis=1))


def energy_weights(Bc, target, w_rs, blend, reg):
    """``solve_energy_weights`` (classical_amg.py:1469-1501) for one row.

    Bc is (m, k): the basis rows picked by the row's column indices, transposed.
    """
    m, k = Bc.shape
    A_ls = np.vstack([Bc, np.ones((1, k))])
    y = np.concatenate([target, [1.0]])
    ATA = A_ls.T @ A_ls + reg * np.eye(k)
    w_ls = np.linalg.solve(ATA, A_ls.T @ y)
    w_ls = np.maximum(w_ls, 0.0)
    s = w_ls.sum()
    if s <= 1e-12:
        return w_rs
    w_ls = w_ls / s
    return (1.0 - blend) * w_rs + blend * w_ls


def prolongation(A, cf_in, strong, basis, blend=0.0, reg=1e-7):
    """``build_prolongation_rs_full`` (classical_amg.py:149-427).

    Returns (P csr, cf after orphan promotion).
    """
    n = A.shape[0]
    r = _row_idx(A)
    col, val = A.indices, A.data
    cf = cf_in.astype(np.int8).copy()
    off = col != r
    diag = np.zeros(n)
    dm = ~off
    np.add.at(diag, r[dm], val[dm])
    diag = np.where(np.abs(diag) > 1e-14, diag, 1.0)
    # orphan promotion (:178-189)
    while True:
        C = cf == 0
        sc = strong & off & C[col]
        cnt = np.bincount(r[sc], minlength=n)
        orphan = (cf == 1) & (cnt == 0)
        if not orphan.any():
            break
        cf[orphan] = 0
    C = cf == 0
    F = ~C
    coarse_nodes = np.nonzero(C)[0]
    f2c = np.full(n, -1, dtype=np.int64)
    f2c[coarse_nodes] = np.arange(len(coarse_nodes))
    sC = strong & off & C[col] & F[r]
    wC = (~strong) & off & C[col] & F[r]
    sF = strong & off & F[col] & F[r]
    wF = (~strong) & off & F[col] & F[r]
    sum_strong = np.zeros(n); np.add.at(sum_strong, r[sC], -val[sC])
    weak_C_sum = np.zeros(n); np.add.at(weak_C_sum, r[wC], -val[wC])
    F_weak_sum = np.zeros(n); np.add.at(F_weak_sum, r[wF], -val[wF])
    cnt = np.bincount(r[sC], minlength=n)
    sc_ptr = np.zeros(n + 1, dtype=np.int64); sc_ptr[1:] = np.cumsum(cnt)
    jc_idx = np.nonzero(sC)[0]
    jc_coarse = f2c[col[jc_idx]]
    den = sum_strong[r[jc_idx]]
    with np.errstate(divide="ignore", invalid="ignore"):
        jc_w = np.where(den > 1e-14, -val[jc_idx] / den, 0.0)
        rows_d = r[sC]
        vals_d = np.nan_to_num(-val[sC] / diag[rows_d], nan=0.0, posinf=0.0, neginf=0.0)
        ff_rows, ff_cols, ff_vals = r[sF], col[sF], val[sF]
        ff_fac = np.nan_to_num(-ff_vals / diag[ff_rows], nan=0.0, posinf=0.0, neginf=0.0)
    cnt_j = cnt[ff_cols]
    den_j = sum_strong[ff_cols]
    valid = (cnt_j > 0) & (den_j > 1e-14)
    rc, cc, vc = [np.zeros(0, np.int64)], [np.zeros(0, np.int64)], [np.zeros(0)]
    if valid.any():
        cv = cnt_j[valid]
        starts = sc_ptr[ff_cols[valid]]
        tot = int(cv.sum())
        base = np.cumsum(cv) - cv
        pos = np.repeat(starts, cv) + (np.arange(tot) - np.repeat(base, cv))
        rc = [np.repeat(ff_rows[valid], cv)]
        cc = [jc_coarse[pos]]
        vc = [np.repeat(ff_fac[valid], cv) * jc_w[pos]]
    inval = ~valid
    if inval.any():
        np.add.at(F_weak_sum, ff_rows[inval], -ff_vals[inval])
    total_weak = weak_C_sum + F_weak_sum
    corr = np.zeros(n)
    mc = (sum_strong > 1e-14) & F
    corr[mc] = total_weak[mc] / sum_strong[mc]
    vals_d = np.maximum(vals_d * (1.0 + corr[rows_d]), 0.0)
    vcon = np.maximum(vc[0], 0.0)
    rows = np.concatenate([coarse_nodes, rows_d, rc[0]])
    cols = np.concatenate([f2c[coarse_nodes], jc_coarse, cc[0]])
    vals = np.concatenate([np.ones(len(coarse_nodes)), vals_d, vcon])
    nc = max(int(f2c.max()) + 1 if len(coarse_nodes) else 1, 1)
    P = sp.coo_matrix((vals, (rows, cols)), shape=(n, nc)).tocsr()
    P.sum_duplicates()
    P.sort_indices()
    # row normalisation of F rows (:334-388)
    rs = np.asarray(P.sum(axis=1)).ravel()
    zero_rows = np.nonzero(F & (rs <= 1e-14))[0]
    if len(zero_rows):
        # injection fallback: first coarse neighbour of the row in A, value 1,
        # placed at the start of the P row
        Pl = P.tolil()
        for node in zero_rows:
            nb = col[A.indptr[node]:A.indptr[node + 1]]
            cn = nb[C[nb]]
            if len(cn) == 0:
                continue
            Pl.rows[node] = [int(f2c[cn[0]])] + list(Pl.rows[node])
            Pl.data[node] = [1.0] + list(Pl.data[node])
        P = sp.csr_matrix(Pl)
        rs = np.asarray(P.sum(axis=1)).ravel()
    scale = np.ones(n)
    mF = F & (rs > 1e-14)
    scale[mF] = 1.0 / rs[mF]
    P.data = np.maximum(P.data * np.repeat(scale, np.diff(P.indptr)), 0.0)
    # energy-minimising blend (:390-419)
    if basis is not None and blend > 0.0:
        Bd = orthonormalize(basis)
        lens = np.diff(P.indptr)
        fr = np.nonzero(F & (lens > 0))[0]
        for k in np.unique(lens[fr]):
            rows_k = fr[lens[fr] == k]
            idx = P.indptr[rows_k][:, None] + np.arange(k)[None, :]
            cols_k = P.indices[idx]                     # (R, k) coarse indices
            Bc = np.transpose(Bd[cols_k], (0, 2, 1))    # fine basis rows at coarse indices
            m = Bc.shape[1]
            A_ls = np.concatenate([Bc, np.ones((len(rows_k), 1, k))], axis=1)
            y = np.concatenate([Bd[rows_k], np.ones((len(rows_k), 1))], axis=1)
            ATA = np.einsum("rmk,rml->rkl", A_ls, A_ls) + reg * np.eye(k)[None]
            rhs = np.einsum("rmk,rm->rk", A_ls, y)
            w_ls = np.maximum(np.linalg.solve(ATA, rhs[..., None])[..., 0], 0.0)
            s = w_ls.sum(axis=1)
            w_rs = P.data[idx]
            ok = s > 1e-12
            w_new = np.where(ok[:, None], (1.0 - blend) * w_rs + blend * (w_ls / np.where(ok, s, 1.0)[:, None]), w_rs)
            P.data[idx] = w_new
            del m
    return P, cf


def truncate_interpolation(P, cf, kmax=0, tf=0.0):
    """Interpolation truncation, an option of the GPU library with no counterpart
    in the reference (restated here as its checker).  Each F row (cf == 1) keeps
    entry e when fewer than ``kmax`` entries outrank it -- a larger weight, or an
    equal weight earlier in the row -- and its weight is at least ``tf`` times
    the row's largest; kept entries are rescaled to the row's old sum.  C rows
    are kept as they are.  ``kmax`` 0 means no cap."""
    P = P.tocsr()
    rows, cols, vals = [], [], []
    for i in range(P.shape[0]):
        a, b = P.indptr[i], P.indptr[i + 1]
        w = P.data[a:b]
        c = P.indices[a:b]
        if cf[i] != 1 or b == a:
            keep = np.ones(b - a, dtype=bool)
            sc = 1.0
        else:
            wmax = w.max()
            keep = w >= tf * wmax
            if kmax > 0:
                order = np.lexsort((np.arange(b - a), -w))   # weight descending, then position
                rank = np.empty(b - a, dtype=np.int64)
                rank[order] = np.arange(b - a)
                keep &= rank < kmax
            kept = w[keep].sum()
            sc = w.sum() / kept if kept > 0.0 else 1.0
        rows.append(np.full(int(keep.sum()), i))
        cols.append(c[keep])
        vals.append(w[keep] * sc)
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    out = sp.csr_matrix((vals, (rows, cols)), shape=P.shape)
    out.sort_indices()
    return out


def galerkin(A, P):
    """``rap_torch`` (classical_amg.py:653-657): A_c = P^T (A P)."""
    Ac = (P.T.tocsr() @ (A @ P)).tocsr()
    Ac.sort_indices()
    return Ac


def inv_relax(A):
    """l1-Jacobi weights (classical_amg.py:885-889): 1/max(|a_ii|, 0.3 sum|a_ij|), <= 1e2."""
    d = np.abs(extract_diag(A))
    ra = np.asarray(abs(A).sum(axis=1)).ravel()
    return np.minimum(1.0 / np.maximum(np.maximum(d, 0.3 * ra), 1e-30), 1e2)


def cheb_lmax(A, inv):
    """Upper bound of the spectrum of diag(inv) A used by the Chebyshev smoother
    (an option of the GPU library; the reference smooths with l1-Jacobi only):
    the Gershgorin bound max_i inv_i * sum_j |a_ij|."""
    ra = np.asarray(abs(A).sum(axis=1)).ravel()
    return float((inv * ra).max()) if A.shape[0] else 0.0


def cheb_smooth(A, inv, lmax, x, b, nu, lower=0.3, zero_x=False):
    """``nu`` steps of the Chebyshev iteration for diag(inv) A on
    [lower * lmax, lmax] (Saad, Iterative Methods for Sparse Linear Systems,
    2nd ed., Alg. 12.1), from x (or from zero): x is updated nu times, with
    nu - 1 products by A after the initial residual.  The GPU kernels follow
    this operation order."""
    theta = 0.5 * (lmax + lower * lmax)
    delta = 0.5 * (lmax - lower * lmax)
    sigma = theta / delta
    rho = 1.0 / sigma
    r = inv * b if zero_x else inv * (b - A @ x)
    d = r / theta
    if zero_x:
        x = np.zeros_like(b)
    for k in range(nu):
        if k == nu - 1:
            x = x + d
            break
        r = r - inv * (A @ d)
        rho_new = 1.0 / (2.0 * sigma - rho)
        d_new = (rho_new * rho) * d + (2.0 * rho_new / delta) * r
        x = x + d
        d, rho = d_new, rho_new
    return x


def equilibrate(A, threshold=1e-6):
    """Equilibration test and scaling (classical_amg.py:763-788, 1334-1355).

    Returns (A_scaled, Dhalf_inv or None).
    """
    d = np.maximum(np.abs(extract_diag(A)), 1e-30)
    med = np.sort(d)[(len(d) - 1) // 2]     # torch.median: lower median
    if med < threshold:
        dh = 1.0 / np.sqrt(d)
        r = _row_idx(A)
        As = A.copy()
        As.data = A.data * dh[r] * dh[A.indices]
        return As, dh
    return A.copy(), None


class AMG:
    """``ClassicalAMG`` (classical_amg.py:694-1392) with a supplied tie-break seed."""

    def __init__(self, A, theta=0.25, max_levels=10, coarsest_size=100, seed=0,
                 nullspace_dim=3, nullspace_blend=0.6, nullspace_reg=1e-6, tiebreaks=None,
                 p_max_elements=0, p_trunc_factor=0.0, smoother="l1jacobi", cheb_lower=0.3,
                 light_sweep_rows=0):
        self.theta, self.max_levels, self.coarsest_size = theta, max_levels, coarsest_size
        # levels of at most this many rows: one sweep before and one after the
        # coarse correction (an option of the GPU library, not the reference's)
        self.light_sweep_rows = int(light_sweep_rows)
        if smoother not in ("l1jacobi", "chebyshev"):
            raise ValueError(f"unknown smoother {smoother!r}")
        self.smoother, self.cheb_lower = smoother, float(cheb_lower)
        self.blend = float(max(0.0, min(1.0, nullspace_blend)))
        self.reg = float(max(1e-10, nullspace_reg))
        A = sp.csr_matrix(A, dtype=np.float64)
        A.sort_indices()
        A, self.Dhalf_inv = equilibrate(A)
        self.levels = []
        basis = nullspace(A.shape[0], nullspace_dim)
        lvl = 0
        for lvl in range(max_levels):
            n = A.shape[0]
            if n <= coarsest_size:
                self.levels.append(dict(A=A, n=n, P=None, inv_relax=inv_relax(A), is_coarsest=True))
                break
            strong = strength(A, theta)
            w = tiebreak(seed, lvl, n) if tiebreaks is None else tiebreaks[lvl]
            cf, n_c = coarsen(A, theta, w)
            if n_c >= n * 0.9:
                self.levels.append(dict(A=A, n=n, P=None, inv_relax=inv_relax(A), is_coarsest=True))
                break
            bl = self.blend if basis is not None else 0.0
            P, cf = prolongation(A, cf, strong, basis, blend=bl, reg=self.reg)
            if p_max_elements > 0 or p_trunc_factor > 0.0:
                P = truncate_interpolation(P, cf, p_max_elements, p_trunc_factor)
            Ac = galerkin(A, P)
            self.levels.append(dict(A=A, n=n, P=P, cf=cf, inv_relax=inv_relax(A), is_coarsest=False))
            if basis is not None:
                basis = orthonormalize(P.T @ basis)
            A = Ac
        if not self.levels or not self.levels[-1]["is_coarsest"]:
            self.levels.append(dict(A=A, n=A.shape[0], P=None, inv_relax=inv_relax(A), is_coarsest=True))

    def update_matrix(self, A):
        """``update_matrix`` (classical_amg.py:1308-1392): frozen P, new Galerkin values."""
        A = sp.csr_matrix(A, dtype=np.float64)
        A.sort_indices()
        A, self.Dhalf_inv = equilibrate(A)
        if A.shape[0] != self.levels[0]["n"]:
            raise ValueError("hierarchy size mismatch")
        self.levels[0]["A"] = A
        self.levels[0]["inv_relax"] = inv_relax(A)
        for l in range(len(self.levels) - 1):
            P = self.levels[l]["P"]
            if P is None:
                continue
            A = galerkin(A, P)
            self.levels[l + 1]["A"] = A
            self.levels[l + 1]["inv_relax"] = inv_relax(A)

    # -------------------------------------------------------------- cycling
    def smooth(self, l, x, b, nu, zero_x=False):
        lv = self.levels[l]
        if getattr(self, "smoother", "l1jacobi") == "chebyshev":
            lmax = cheb_lmax(lv["A"], lv["inv_relax"])
            return cheb_smooth(lv["A"], lv["inv_relax"], lmax, x, b, nu, self.cheb_lower, zero_x)
        for _ in range(nu):
            x = x + 0.7 * lv["inv_relax"] * (b - lv["A"] @ x)
        return x

    def coarse_solve(self, lv, b):
        """Coarsest level (classical_amg.py:1045-1069): pin DOF 0, dense solve."""
        n = lv["n"]
        bl = b.copy()
        if n > 0:
            bl[0] = 0.0
        if n <= 500:
            Ad = lv["A"].toarray()
            if n > 0:
                Ad[0, :] = 0.0
                Ad[:, 0] = 0.0
                Ad[0, 0] = 1.0
            try:
                return np.linalg.solve(Ad, bl)
            except np.linalg.LinAlgError:
                return np.linalg.lstsq(Ad, bl, rcond=None)[0]
        x = np.zeros_like(bl)
        for _ in range(50):
            x = x + 0.7 * lv["inv_relax"] * (bl - lv["A"] @ x)
        return x

    def vcycle(self, l, x, b, pre=3, post=2):
        """``_v_cycle`` (classical_amg.py:1037-1106)."""
        lv = self.levels[l]
        if lv["is_coarsest"]:
            return self.coarse_solve(lv, b)
        light = lv["n"] <= getattr(self, "light_sweep_rows", 0)
        x = self.smooth(l, x, b, 1 if light else pre, zero_x=(l > 0 or not np.any(x)))
        r = b - lv["A"] @ x
        rc = lv["P"].T @ r
        ec = self.vcycle(l + 1, np.zeros_like(rc), rc, pre, post)
        x = x + lv["P"] @ ec
        return self.smooth(l, x, b, 1 if light else post)

    def solve(self, b, x0=None, tol=1e-6, max_iter=10):
        """``ClassicalAMG.solve`` (classical_amg.py:1108-1155). Returns (x, cycles, rel_res)."""
        if self.Dhalf_inv is not None:
            bs = self.Dhalf_inv * b
            xs = np.zeros_like(bs) if x0 is None else x0 / self.Dhalf_inv
        else:
            bs = b.copy()
            xs = np.zeros_like(b) if x0 is None else x0.copy()
        bn = np.linalg.norm(bs)
        rel, cyc = np.inf, 0
        for cyc in range(1, max_iter + 1):
            xs = self.vcycle(0, xs, bs)
            rel = np.linalg.norm(bs - self.levels[0]["A"] @ xs) / (bn + 1e-30)
            if rel < tol:
                break
        x = self.Dhalf_inv * xs if self.Dhalf_inv is not None else xs
        return x, cyc, rel

    def apply(self, b, cycles=1, apply_tol=5e-2, apply_max_cycles=8):
        """``ClassicalAMG.apply`` (classical_amg.py:1157-1180)."""
        bs = self.Dhalf_inv * b if self.Dhalf_inv is not None else b.copy()
        xs = np.zeros_like(bs)
        bn = np.linalg.norm(bs)
        cyc = 0
        while cyc < apply_max_cycles:
            xs = self.vcycle(0, xs, bs)
            cyc += 1
            rel = np.linalg.norm(bs - self.levels[0]["A"] @ xs) / (bn + 1e-30)
            if cyc >= cycles and rel < apply_tol:
                break
        return self.Dhalf_inv * xs if self.Dhalf_inv is not None else xs


class AMGSolver:
    """``amg_solve`` (pressure_amg.py:35-89): cached hierarchy, ``update_matrix`` on a hit."""

    def __init__(self, tol=1e-6, max_cycles=20, theta=0.25, max_levels=10, coarsest_size=200, seed=0):
        self.kw = dict(theta=theta, max_levels=max_levels, coarsest_size=coarsest_size, seed=seed)
        self.tol, self.max_cycles = tol, max_cycles
        self.cache = {}
        self.history = []

    def __call__(self, A, b):
        key = (A.shape, self.kw["theta"], self.kw["max_levels"], self.kw["coarsest_size"])
        amg = self.cache.get(key)
        if amg is None:
            amg = AMG(A, **self.kw)
            self.cache[key] = amg
        else:
            amg.update_matrix(A)
        x, cyc, rel = amg.solve(b, tol=self.tol, max_iter=self.max_cycles)
        self.history.append((cyc, rel))
        return x
