"""PPO rollout collection with the environment step inside a CUDA graph.

Counterpart of the sampling loop of the reference's PPO
(``rl/ppo.py:247-300``): per step, the policy samples actions and values,
the vec-env steps, time-outs are bootstrapped with the value of the final
observation (``rewards += gamma V(final_obs)``), and the transition is
stored; after ``steps`` steps the GAE advantages are computed
(``rl/common/memory.py``).  Here one whole rollout step -- policy forward,
Gaussian sampling, action clipping, the env step (itself a graph: prologue,
batched integration, fused reward/termination/reset epilogue), the bootstrap
and the stores -- is captured once into a CUDA graph and replayed
``steps`` times; the buffer slot is a device counter, so nothing on the host
changes between replays and a rollout is ``steps`` graph launches with no
host synchronisation.

The policy is a small actor-critic MLP (Gaussian actions with a learned
log-std), written here; training (the PPO update) is outside this module.
"""
from __future__ import annotations

from typing import Dict, Optional

import torch
from torch import nn


class ActorCritic(nn.Module):
    def __init__(self, obs_dim: int, act_dim: int, hidden: int = 64, log_std: float = -0.5):
        super().__init__()
        self.actor = nn.Sequential(nn.Linear(obs_dim, hidden), nn.Tanh(), nn.Linear(hidden, hidden), nn.Tanh(),
                                   nn.Linear(hidden, act_dim))
        self.critic = nn.Sequential(nn.Linear(obs_dim, hidden), nn.Tanh(), nn.Linear(hidden, hidden), nn.Tanh(),
                                    nn.Linear(hidden, 1))
        self.log_std = nn.Parameter(torch.full((act_dim,), float(log_std)))

    def value(self, obs: torch.Tensor) -> torch.Tensor:
        return self.critic(obs).squeeze(-1)

    def sample(self, obs: torch.Tensor):
        mean = self.actor(obs)
        std = self.log_std.exp()
        a = mean + std * torch.randn_like(mean)
        logp = (-0.5 * ((a - mean) / std) ** 2 - self.log_std - 0.9189385332046727).sum(-1)
        return a, logp, self.value(obs)


class GraphedRollout:
    """Collects ``steps`` transitions of every env of ``env``
    (``CKM1DVecEnv``) with one CUDA-graph replay per step."""

    def __init__(self, env, policy: ActorCritic, steps: int, gamma: float = 0.99, gae_lambda: float = 0.95,
                 action_low: float = 0.0, action_high: float = 1.5):
        self.env, self.policy = env, policy
        self.steps, self.gamma, self.lam = int(steps), float(gamma), float(gae_lambda)
        self.lo, self.hi = float(action_low), float(action_high)
        n, obs_dim = env.obs.shape
        act_dim = env.actions.shape[1]
        dev = env.obs.device
        f32 = torch.float32
        self.buf: Dict[str, torch.Tensor] = {
            "obs": torch.zeros((self.steps, n, obs_dim), dtype=f32, device=dev),
            "actions": torch.zeros((self.steps, n, act_dim), dtype=f32, device=dev),
            "logprobs": torch.zeros((self.steps, n), dtype=f32, device=dev),
            "values": torch.zeros((self.steps, n), dtype=f32, device=dev),
            "rewards": torch.zeros((self.steps, n), dtype=f32, device=dev),      # bootstrapped
            "raw_rewards": torch.zeros((self.steps, n), dtype=f32, device=dev),
            "dones": torch.zeros((self.steps, n), dtype=f32, device=dev),
        }
        self.t = torch.zeros(1, dtype=torch.long, device=dev)
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _step(self) -> None:
        env, b, t = self.env, self.buf, self.t
        obs = env.obs
        a, logp, v = self.policy.sample(obs)
        b["obs"].index_copy_(0, t, obs.unsqueeze(0))
        b["actions"].index_copy_(0, t, a.unsqueeze(0))
        b["logprobs"].index_copy_(0, t, logp.unsqueeze(0))
        b["values"].index_copy_(0, t, v.unsqueeze(0))
        env.actions.copy_(a.clamp(self.lo, self.hi))
        env.step_physics()
        r = env.rewards
        tout = env.time_outs.to(torch.float32)
        boot = r + self.gamma * self.policy.value(env.final_obs) * tout
        b["rewards"].index_copy_(0, t, boot.unsqueeze(0))
        b["raw_rewards"].index_copy_(0, t, r.unsqueeze(0))
        b["dones"].index_copy_(0, t, env.done.to(torch.float32).unsqueeze(0))
        t.add_(1)

    def capture(self) -> None:
        """Warm-up on a side stream, then capture one rollout step."""
        with torch.no_grad():
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                self._step()            # a real step (advances the envs once), as capture warm-up
            torch.cuda.current_stream().wait_stream(side)
            self.t.zero_()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._step()
        self.t.zero_()

    def collect(self) -> Dict[str, torch.Tensor]:
        """One rollout: `steps` graph replays, then GAE advantages and returns."""
        if self.graph is None:
            self.capture()
        self.t.zero_()
        for _ in range(self.steps):
            self.graph.replay()
        with torch.no_grad():
            last_v = self.policy.value(self.env.obs)
        b = self.buf
        adv = torch.zeros_like(b["rewards"])
        gae = torch.zeros_like(last_v)
        for s in reversed(range(self.steps)):
            nxt = last_v if s == self.steps - 1 else b["values"][s + 1]
            nonterm = 1.0 - b["dones"][s]
            delta = b["rewards"][s] + self.gamma * nxt * nonterm - b["values"][s]
            gae = delta + self.gamma * self.lam * nonterm * gae
            adv[s] = gae
        out = dict(b)
        out["advantages"] = adv
        out["returns"] = adv + b["values"]
        return out
