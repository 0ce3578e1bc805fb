"""``ReservoirEnv`` (src/rl_env.py) with its time step on the B200, and a batched
form that advances many environments together.

``ReservoirEnv`` keeps the reference's constructor, ``reset``/``step``/``render``
and its action, observation and reward definitions (rl_env.py:14-152).  It is a
``gymnasium.Env`` when gymnasium is importable; otherwise it exposes the same
methods and ``action_space``/``observation_space`` as plain shape records.

``ReservoirVecEnv`` holds several environments (one config each, or copies) and
advances all of them with one ``impes_ensemble_run`` call per ``step``: each
environment keeps its own model and hierarchy, so its trajectory equals the
single environment's.  A member whose pressure solve misses its tolerance ends
its episode with the reference's -1e3 reward (rl_env.py:97-100); the batched
step solves the pressure with FGMRES and the AMG V-cycle (the ensemble driver)
whatever ``pressure_solver`` says, and does not retry with a smaller dt.
"""
from __future__ import annotations

import json
from types import SimpleNamespace
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .ensemble import Ensemble
from .simulator import Fluid, Reservoir, Simulator, WellManager

try:  # the reference's base class, when available
    import gymnasium as _gym
    from gymnasium import spaces as _spaces
    _Base = _gym.Env
except ImportError:  # pragma: no cover - depends on the environment
    _gym, _spaces, _Base = None, None, object

__all__ = ["ReservoirEnv", "ReservoirVecEnv"]


def _box(low, high, shape):
    if _spaces is not None:
        return _spaces.Box(low=low, high=high, shape=shape, dtype=np.float32)
    return SimpleNamespace(low=low, high=high, shape=shape, dtype=np.float32)


def _apply_action(wells, action):
    """rl_env.py:127-140: rate wells change by up to +-20 %, BHP wells by +-5 MPa."""
    for a, well in zip(action, wells):
        if well.control_type == "rate":
            base = well.control_value
            well.control_value = float(base + base * 0.2 * a)
        elif well.control_type == "bhp":
            well.control_value = float(well.control_value + 5.0 * a)


class ReservoirEnv(_Base):
    metadata = {"render_modes": ["human"], "render_fps": 4}

    def __init__(self, config_path: str, max_steps: int = 365, device: Optional[torch.device] = None,
                 render_mode: Optional[str] = None) -> None:
        if _Base is not object:
            super().__init__()
        self.config_path = config_path
        self.max_steps = max_steps
        self.render_mode = render_mode
        self.device = device or torch.device("cuda")
        self._build()
        n_wells = len(self.well_manager.wells)
        self.action_space = _box(-1.0, 1.0, (n_wells,))
        nx, ny, nz = self.reservoir.dimensions
        self.observation_space = _box(-np.inf, np.inf, (nx * ny * nz * 2,))
        self._step_count = 0
        self._prev_oil_mass = self._calc_oil_mass().item()

    def _build(self):
        with open(self.config_path, "r", encoding="utf-8") as f:
            cfg = json.load(f)
        self.cfg = cfg
        self.reservoir = Reservoir(cfg["reservoir"], device=self.device)
        self.well_manager = WellManager(cfg["wells"], self.reservoir)
        self.fluid = Fluid(cfg["fluid"], self.reservoir, device=self.device)
        self.simulator = Simulator(reservoir=self.reservoir, fluid=self.fluid, well_manager=self.well_manager,
                                   sim_params=cfg.get("simulation", {}), device=self.device)

    # Gym API (rl_env.py:63-115)
    def reset(self, *, seed: Optional[int] = None, options: Optional[Dict] = None):
        if _Base is not object:
            super().reset(seed=seed)
        self.simulator.close()
        self._build()
        self._step_count = 0
        self._prev_oil_mass = self._calc_oil_mass().item()
        return self._get_observation(), {}

    def step(self, action: np.ndarray) -> Tuple[np.ndarray, float, bool, bool, Dict]:
        _apply_action(self.well_manager.wells, action)
        dt_sec = self.simulator.sim_params.get("time_step_days", 1.0) * 24 * 3600
        if not self.simulator.run_step(dt_sec):
            return self._get_observation(), -1e3, True, False, {"converged": False}
        return self._after_step()

    def _after_step(self):
        self._step_count += 1
        obs = self._get_observation()
        reward = self._calc_reward()
        return obs, reward, self._step_count >= self.max_steps, False, {"converged": True}

    def render(self, mode: str = "human"):
        if mode != "human":
            raise NotImplementedError
        print(f"mean pressure: {float(self.fluid.pressure.mean() / 1e6):.2f} MPa, step {self._step_count}")

    def close(self):
        self.simulator.close()

    # rl_env.py:121-152
    def _get_observation(self) -> np.ndarray:
        p = self.fluid.pressure.cpu().numpy().flatten() / 1e7
        sw = self.fluid.s_w.cpu().numpy().flatten()
        return np.concatenate([p, sw]).astype(np.float32)

    def _calc_oil_mass(self) -> torch.Tensor:
        phi = self.reservoir.porosity
        s_o = self.fluid.s_o.reshape(phi.shape)
        return torch.sum(phi * s_o * self.fluid.rho_o.reshape(phi.shape) * self.reservoir.cell_volume)

    def _calc_reward(self) -> float:
        oil_mass = self._calc_oil_mass().item()
        produced = self._prev_oil_mass - oil_mass
        self._prev_oil_mass = oil_mass
        return produced / 1e6


class ReservoirVecEnv:
    """``len(config_paths)`` environments stepped together on one GPU."""

    def __init__(self, config_paths: Sequence[str], max_steps: int = 365,
                 device: Optional[torch.device] = None, workers: int = 8):
        self.envs = [ReservoirEnv(p, max_steps=max_steps, device=device) for p in config_paths]
        dts = {e.simulator.sim_params.get("time_step_days", 1.0) for e in self.envs}
        if len(dts) != 1:
            raise ValueError("all environments of a batch need the same time_step_days")
        self.dt_sec = dts.pop() * 24 * 3600
        self.workers = workers
        self.done = [False] * len(self.envs)

    def reset(self):
        out = [e.reset() for e in self.envs]
        self.done = [False] * len(self.envs)
        return [o for o, _ in out], [i for _, i in out]

    def _ensemble(self, idx):
        ens = Ensemble.__new__(Ensemble)
        ens.device = self.envs[0].device
        ens.sims = [self.envs[i].simulator for i in idx]
        for sim in ens.sims:
            sim._ensure_amg()
        ens.members = list(idx)
        ens.cells = [int(np.prod(e.reservoir.dimensions)) for e in self.envs]
        ens.workers = self.workers
        ens.last_stats, ens.last_span_ms = [], 0.0
        return ens

    def step(self, actions):
        """One step of every environment that is not done; returns lists of
        (obs, reward, terminated, truncated, info)."""
        idx = [i for i, d in enumerate(self.done) if not d]
        for i in idx:
            _apply_action(self.envs[i].well_manager.wells, actions[i])
            self.envs[i].simulator._set_well_cells()
        ens = self._ensemble(idx)
        try:
            ens.run(1, self.dt_sec)
        except _lib.ImpesError:
            pass                       # per-member statuses below
        status = {s["member"]: s["status"] for s in ens.last_stats}
        res = []
        for i, e in enumerate(self.envs):
            if i not in status:
                res.append((e._get_observation(), 0.0, True, False, {"converged": False, "done": True}))
            elif status[i] != 0:
                self.done[i] = True
                res.append((e._get_observation(), -1e3, True, False, {"converged": False}))
            else:
                r = e._after_step()
                self.done[i] = r[2]
                res.append(r)
        return tuple(list(x) for x in zip(*res))

    def close(self):
        for e in self.envs:
            e.close()
