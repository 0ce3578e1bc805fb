"""The ReservoirEnv mirror (src/rl_env.py) and its batched form."""
import json

import numpy as np
import pytest

from impes_b200 import scenarios

pytestmark = pytest.mark.gpu


def _config(tmp_path, seed, nx=12, ny=10, nz=2):
    cfg, f = scenarios.two_phase_2d(seed=seed, nx=nx, ny=ny, nz=nz, steps=4, sigma=0.0)
    cfg["simulation"]["amg"].update({"tol": 1e-10, "norm": "jacobi"})
    path = tmp_path / f"env{seed}.json"
    path.write_text(json.dumps(cfg))
    return str(path)


def test_env_step_reward_and_controls(tmp_path):
    from impes_b200.rl_env import ReservoirEnv
    env = ReservoirEnv(_config(tmp_path, 0), max_steps=3)
    obs, info = env.reset()
    assert obs.shape == env.observation_space.shape and obs.dtype == np.float32
    inj = env.well_manager.wells[0]
    q0 = inj.control_value
    obs, reward, term, trunc, info = env.step(np.array([1.0, -1.0], dtype=np.float32))
    assert info["converged"] and not term and np.isfinite(reward)
    assert inj.control_value == pytest.approx(q0 * 1.2)
    assert env.well_manager.wells[1].control_value == pytest.approx(15.0 - 5.0)
    # the new controls reach the device: a different action gives a different state
    env2 = ReservoirEnv(_config(tmp_path, 0), max_steps=3)
    obs2, *_ = env2.step(np.array([0.0, 0.0], dtype=np.float32))
    assert not np.array_equal(obs, obs2)
    for _ in range(2):
        obs, reward, term, trunc, info = env.step(np.zeros(2, dtype=np.float32))
    assert term
    env.close()
    env2.close()


def test_vector_env_equals_single_envs(tmp_path):
    from impes_b200.rl_env import ReservoirEnv, ReservoirVecEnv
    paths = [_config(tmp_path, s, nx=8 + 4 * s) for s in range(3)]
    cfg0 = json.loads(open(paths[0]).read())
    assert cfg0["simulation"]["pressure_solver"] == "gmres_amg"
    venv = ReservoirVecEnv(paths, max_steps=5, workers=2)
    venv.reset()
    rng = np.random.default_rng(1)
    acts = [rng.uniform(-1, 1, size=(3, 2)).astype(np.float32) for _ in range(2)]
    for a in acts:
        obs, rew, term, trunc, info = venv.step(a)
        assert all(i["converged"] for i in info)
    for k, p in enumerate(paths):
        env = ReservoirEnv(p, max_steps=5)
        for a in acts:
            o, r, *_ = env.step(a[k])
        assert np.array_equal(o, obs[k])
        assert r == pytest.approx(rew[k], rel=1e-12, abs=1e-15)
        env.close()
    venv.close()
