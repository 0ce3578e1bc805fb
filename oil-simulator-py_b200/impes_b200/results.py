"""Result files of a full run, as the reference's ``Simulator.run`` writes them
(simulation.py:2121-2260): a directory ``results/<name>_<timestamp>/`` holding
``<name>.txt`` (final-state summary and mass-balance block, optionally the full
arrays) and ``<name>.npz`` (keys ``pressure``, ``sw``, ``sg``, ``so``).

Intermediate states are written every ``save_interval`` steps, at the
reference's cadence (:2182-2192), as ``intermediate/<name>_step_<i>.npz`` with
``pressure``, ``sw``, ``sg`` -- the reference renders PNG plots there; plotting
is not part of this package.
"""
from __future__ import annotations

import datetime
import os

import numpy as np

__all__ = ["results_dir", "write_summary", "write_npz", "write_snapshot"]


def results_dir(output_filename: str, root: str = "results", stamp: str | None = None) -> str:
    """``results/<name>_<YYYYmmdd_HHMMSS>`` (simulation.py:2150-2153), created."""
    stamp = stamp or datetime.datetime.now().strftime("%Y%m%d_%H%M%S")
    d = os.path.join(root, f"{output_filename}_{stamp}")
    os.makedirs(d, exist_ok=True)
    return d


def write_summary(path: str, p, sw, sg, so, mass_balance: dict, full_arrays: bool = False) -> None:
    """The summary text file of simulation.py:2212-2241, line for line."""
    p, sw, sg, so = (np.asarray(a) for a in (p, sw, sg, so))
    mb = mass_balance
    with open(path, "w") as f:
        f.write("=== SUMMARY (final) ===\n")
        f.write(f"Pressure MPa: min={p.min()/1e6:.2f}, max={p.max()/1e6:.2f}, mean={p.mean()/1e6:.2f}\n")
        f.write(f"Sw: min={sw.min():.4f}, max={sw.max():.4f}, mean={sw.mean():.4f}\n")
        f.write(f"Sg: min={sg.min():.4f}, max={sg.max():.4f}, mean={sg.mean():.4f}\n")
        f.write(f"So: min={so.min():.4f}, max={so.max():.4f}, mean={so.mean():.4f}\n")
        net_w = mb["water"]["in"] - mb["water"]["out"]
        net_g = mb["gas"]["in"] - mb["gas"]["out"]
        net_o = mb["oil"]["in"] - mb["oil"]["out"]
        f.write("\n=== MASS BALANCE (kg) ===\n")
        f.write(f"water: in={mb['water']['in']:.6e}, out={mb['water']['out']:.6e}, net={net_w:.6e}\n")
        f.write(f"gas:   in={mb['gas']['in']:.6e}, out={mb['gas']['out']:.6e}, net={net_g:.6e}\n")
        f.write(f"oil:   in={mb['oil']['in']:.6e}, out={mb['oil']['out']:.6e}, net={net_o:.6e}\n")
        f.write(f"total net={net_w+net_g+net_o:.6e}\n")
        if full_arrays:
            f.write("\n\nFinal Pressure (MPa):\n")
            f.write(np.array2string(p / 1e6, threshold=np.inf, formatter={"float_kind": lambda x: "%.2f" % x}))
            f.write("\n\nFinal Water Saturation:\n")
            f.write(np.array2string(sw, threshold=np.inf, formatter={"float_kind": lambda x: "%.4f" % x}))
            f.write("\n\nFinal Gas Saturation:\n")
            f.write(np.array2string(sg, threshold=np.inf, formatter={"float_kind": lambda x: "%.4f" % x}))
            f.write("\n\nFinal Oil Saturation:\n")
            f.write(np.array2string(so, threshold=np.inf, formatter={"float_kind": lambda x: "%.4f" % x}))


def write_npz(path: str, p, sw, sg, so) -> None:
    """Final fields (simulation.py:2245-2248)."""
    np.savez_compressed(path, pressure=np.asarray(p), sw=np.asarray(sw), sg=np.asarray(sg), so=np.asarray(so))


def write_snapshot(path: str, p, sw, sg) -> None:
    np.savez_compressed(path, pressure=np.asarray(p), sw=np.asarray(sw), sg=np.asarray(sg))
