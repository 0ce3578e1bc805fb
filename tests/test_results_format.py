"""Result files in the reference's layout (simulation.py:2207-2248)."""
import os

import numpy as np

from impes_b200.results import results_dir, write_npz, write_summary


def _expected(p, sw, sg, so, mb):
    net_w = mb["water"]["in"] - mb["water"]["out"]
    net_g = mb["gas"]["in"] - mb["gas"]["out"]
    net_o = mb["oil"]["in"] - mb["oil"]["out"]
    return ("=== SUMMARY (final) ===\n"
            f"Pressure MPa: min={p.min()/1e6:.2f}, max={p.max()/1e6:.2f}, mean={p.mean()/1e6:.2f}\n"
            f"Sw: min={sw.min():.4f}, max={sw.max():.4f}, mean={sw.mean():.4f}\n"
            f"Sg: min={sg.min():.4f}, max={sg.max():.4f}, mean={sg.mean():.4f}\n"
            f"So: min={so.min():.4f}, max={so.max():.4f}, mean={so.mean():.4f}\n"
            "\n=== MASS BALANCE (kg) ===\n"
            f"water: in={mb['water']['in']:.6e}, out={mb['water']['out']:.6e}, net={net_w:.6e}\n"
            f"gas:   in={mb['gas']['in']:.6e}, out={mb['gas']['out']:.6e}, net={net_g:.6e}\n"
            f"oil:   in={mb['oil']['in']:.6e}, out={mb['oil']['out']:.6e}, net={net_o:.6e}\n"
            f"total net={net_w+net_g+net_o:.6e}\n")


def test_summary_and_npz_layout(tmp_path):
    rng = np.random.default_rng(0)
    shape = (4, 3, 2)
    p = 2e7 + 1e6 * rng.random(shape)
    sw = 0.2 + 0.5 * rng.random(shape)
    sg = 0.1 * rng.random(shape)
    so = 1.0 - sw - sg
    mb = {"water": {"in": 1.5e4, "out": 2.0e3}, "oil": {"in": 0.0, "out": 7.7e3},
          "gas": {"in": 12.0, "out": 0.5}}
    d = results_dir("case", root=str(tmp_path), stamp="20260101_000000")
    assert d == os.path.join(str(tmp_path), "case_20260101_000000") and os.path.isdir(d)
    write_summary(os.path.join(d, "case.txt"), p, sw, sg, so, mb)
    with open(os.path.join(d, "case.txt")) as f:
        assert f.read() == _expected(p, sw, sg, so, mb)
    write_summary(os.path.join(d, "full.txt"), p, sw, sg, so, mb, full_arrays=True)
    with open(os.path.join(d, "full.txt")) as f:
        txt = f.read()
    assert txt.startswith(_expected(p, sw, sg, so, mb)) and "Final Oil Saturation:" in txt
    write_npz(os.path.join(d, "case.npz"), p, sw, sg, so)
    z = np.load(os.path.join(d, "case.npz"))
    assert sorted(z.files) == ["pressure", "sg", "so", "sw"]
    assert np.array_equal(z["pressure"], p) and z["sw"].shape == shape
