"""Batched control environment over the ensemble stepper.

Each instance of a qaf.Ensemble is one environment of the active-nematic
flow (the friction solver of InertialFriction/friction/friction.cu): an action
sets the instance's activity Ra (and, optionally, its friction Rf) for the
next `steps_per_action` IF-RK4 steps; an observation is the instance's
(energy, enstrophy) after them (qaf_ensemble_diagnostics); the default reward
is minus the enstrophy. All instances step together in one CUDA graph launch
per step. The reference has no such interface (its README lists a Python
interface as to be done).

    env = qaf.env.EnsembleEnv([128] * 64, qaf.Params(dt=1e-3), lx=16 * math.pi)
    obs = env.reset(seeds=range(64))                 # [64, 2] float64 (energy, enstrophy)
    obs, reward, info = env.step(alpha)              # alpha: 64 activities
"""
from __future__ import annotations

import math
from typing import Callable, Optional, Sequence

from . import F32, Ensemble, Params


class EnsembleEnv:
    def __init__(self, sizes: Sequence[int], params: Params, lx: float = 16 * math.pi, dtype: int = F32,
                 steps_per_action: int = 10, rf: Optional[Sequence[float]] = None, tune: bool = False,
                 reward: Optional[Callable] = None):
        self.sizes = [int(n) for n in sizes]
        self.params = params
        self.steps_per_action = int(steps_per_action)
        if self.steps_per_action < 1:
            raise ValueError("steps_per_action must be >= 1")
        k = len(self.sizes)
        self.rf = [float(params.rf)] * k if rf is None else [float(v) for v in rf]
        self.alpha = [float(params.alpha)] * k
        self.ens = Ensemble(self.sizes, params, self.alpha, self.rf, lx=lx, dtype=dtype, tune=tune)
        self.reward_fn = reward if reward is not None else (lambda obs: -obs[:, 1])
        self.t = 0

    def __len__(self):
        return len(self.sizes)

    def _obs_initial(self):
        import torch
        out = torch.empty((len(self.sizes), 2), dtype=torch.float64)
        for k in range(len(self.sizes)):
            m = self.ens.mesh(k)
            w, _, _ = self.ens.store(k)
            e, z, _ = m.diagnostics(w)
            out[k, 0], out[k, 1] = e, z
        return out

    def reset(self, seeds: Sequence[int], lo: float = -0.01, hi: float = 0.01):
        """Seeded random Q, w = 0, activity back to params.alpha; returns the observation [n, 2]."""
        seeds = [int(s) for s in seeds]
        if len(seeds) != len(self.sizes):
            raise ValueError("one seed per instance")
        self.alpha = [float(self.params.alpha)] * len(self.sizes)
        self.ens.set_controls(self.alpha, self.rf)
        self.ens.init_random(seeds, lo, hi)
        self.t = 0
        return self._obs_initial()

    def step(self, alpha: Sequence[float], rf: Optional[Sequence[float]] = None):
        """Apply the activities (and frictions) for steps_per_action steps; returns (obs, reward, info)."""
        import torch
        alpha = [float(v) for v in alpha]
        if len(alpha) != len(self.sizes):
            raise ValueError("one action per instance")
        if not all(math.isfinite(v) for v in alpha):
            raise ValueError("non-finite action")
        self.alpha = alpha
        if rf is not None:
            self.rf = [float(v) for v in rf]
        self.ens.set_controls(self.alpha, self.rf)
        self.ens.advance(self.steps_per_action)
        self.t += self.steps_per_action
        obs = torch.tensor(self.ens.diagnostics(), dtype=torch.float64)
        return obs, self.reward_fn(obs), {"t": self.t, "alpha": list(self.alpha)}

    def vorticity(self, k: int):
        """The physical vorticity field of instance k (ny x nx), for richer observations."""
        m = self.ens.mesh(k)
        w, _, _ = self.ens.store(k)
        return m.bwd_trans(w)
