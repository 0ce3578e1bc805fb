"""Helpers shared by the GPU parity tests."""
import json

import numpy as np
import scipy.sparse as sp

from oracle.impes import Model


def fixture_fields(g):
    """The rock fields of a fixture: stored in it, or (long-run fixtures) rebuilt
    by the scenario call it names and checked against its stored digest."""
    if "kx" in g:
        return {k: g[k] for k in ("kx", "ky", "kz", "poro")}
    import hashlib
    from impes_b200 import scenarios
    gen = json.loads(str(g["fields_generator"]))
    _, f = getattr(scenarios, gen["scenario"])(**gen["kwargs"])
    f = {k: np.ascontiguousarray(f[k], dtype=np.float64) for k in ("kx", "ky", "kz", "poro")}
    h = hashlib.sha256()
    for k in ("kx", "ky", "kz", "poro"):
        h.update(f[k].tobytes())
    assert h.hexdigest() == str(g["fields_sha256"]), "scenario fields differ from the fixture's"
    return f


def cfg_fields(g):
    cfg = json.loads(str(g["cfg"]))
    return cfg, fixture_fields(g)


def oracle_model(g):
    cfg, f = cfg_fields(g)
    return Model(cfg, f["kx"], f["ky"], f["kz"], f["poro"])


def gpu_sim(cfg, fields, **amg):
    from impes_b200.simulator import build_from_config
    cfg = json.loads(json.dumps(cfg))
    # the FGMRES solver unless the configuration names one (the drop-in default
    # is the reference's own Jacobi-PCG)
    cfg.setdefault("simulation", {}).setdefault("pressure_solver", "gmres_amg")
    cfg["simulation"].setdefault("amg", {}).update(amg)
    return build_from_config(cfg, fields, device="cuda")


def to_np(t):
    return t.detach().reshape(-1).cpu().numpy()


def rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def csr_from(rowptr, col, val, n, m=None):
    return sp.csr_matrix((to_np(val) if hasattr(val, "cpu") else val,
                          to_np(col) if hasattr(col, "cpu") else col,
                          to_np(rowptr) if hasattr(rowptr, "cpu") else rowptr), shape=(n, m or n))
