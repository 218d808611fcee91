"""qaf.env.EnsembleEnv: the batched control interface over the ensemble stepper."""
import math

import pytest

pytestmark = pytest.mark.gpu


def test_reset_and_step_match_the_ensemble(cuda):
    import torch

    import qaf
    import qaf.env as QE
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=1e-3)
    sizes = [64, 64, 128]
    env = QE.EnsembleEnv(sizes, p, lx=16 * math.pi, steps_per_action=5)
    obs0 = env.reset([1, 2, 3])
    assert obs0.shape == (3, 2) and bool(torch.all(obs0 == 0))      # the initial state has w = 0
    actions = [0.5, 1.5, 1.0]
    obs, reward, info = env.step(actions)
    assert obs.shape == (3, 2) and torch.equal(reward, -obs[:, 1]) and info["t"] == 5
    assert bool(torch.all(obs[:, 1] > 0))
    # the same through the ensemble API directly
    ens = qaf.Ensemble(sizes, p, [1.0] * 3, [0.1] * 3, lx=16 * math.pi)
    ens.init_random([1, 2, 3])
    ens.set_controls(actions)
    ens.advance(5)
    ref = torch.tensor(ens.diagnostics(), dtype=torch.float64)
    assert torch.allclose(obs, ref, rtol=1e-12, atol=0)              # the sums use atomics
    for k in range(3):
        for x, y in zip(env.ens.store(k), ens.store(k)):
            assert torch.equal(x, y)
    # reset restores the initial observation
    again = env.reset([1, 2, 3])
    assert torch.equal(again, obs0)
    assert env.vorticity(2).shape == (128, 128)


def test_invalid_actions(cuda):
    import qaf
    import qaf.env as QE
    env = QE.EnsembleEnv([64, 64], qaf.Params(dt=1e-3), lx=16 * math.pi)
    env.reset([1, 2])
    with pytest.raises(ValueError):
        env.step([1.0])
    with pytest.raises(ValueError):
        env.step([1.0, float("nan")])
    with pytest.raises(ValueError):
        env.reset([1])
