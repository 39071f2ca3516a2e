"""GPU-resident vectorised bubble position-control environment.

B200 counterpart of the reference's ``PosNBC1D``
(``coupledbubble_control/envs/bubble_1D_pos_control.py``): N coupled bubbles
per environment, the acoustic amplitudes (PA_1, PA_2) as the action, bubble
positions and radii as the observation, target positions, reward and
termination as in the reference (``get_rewards`` :792-813,
``check_termination`` :772-789, ``advance_time`` :816-826,
``final_termination`` :830-853), and random scene resets
(``SceneGenerator._random_uniform_position_1D`` :176-234).

One ``step`` is one CUDA-graph launch (``cbc_env_plan_create``): action ->
control parameters, time reset, the batched integration of ``time_step_length``
periods for every env, and the float32 observation written straight into
``self.obs`` (a torch tensor the caller can keep; no copy).  The state stays
on the device between steps.  Reward, termination and resets are a handful of
torch ops on the same stream.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Tuple

import numpy as np

from .. import _lib, scenes
from ..ensemble import Ensemble, make_work_list
from ..models import SolverSpec


class SceneGenerator:
    """Random chains of bubbles inside [domain_min + margin, domain_max - margin]
    with neighbour gaps in [min_distance, max_distance] (reference
    SceneGenerator, envs/bubble_1D_pos_control.py:46-249, 'random' positions,
    'center' alignment)."""

    def __init__(self, num_bubbles: int, min_distance: float = 0.05, max_distance: float = 0.9,
                 margin: float = 0.05, domain_min: float = -0.5, domain_max: float = 0.5, seed: int = 42,
                 device="cuda"):
        import torch
        self.K = num_bubbles
        self.min_distance, self.max_distance = min_distance, max_distance
        self.lo, self.hi = domain_min + margin, domain_max - margin
        self.gen = torch.Generator(device=device)
        self.gen.manual_seed(seed)
        self.device = device
        avail = self.hi - self.lo
        if (self.K - 1) * min_distance > avail:
            raise ValueError(f"Cannot fit: the scene needs {(self.K - 1) * min_distance:.2f}, domain is {avail:.2f}")

    def positions(self, n: int, dtype=None):
        import torch
        dtype = dtype or torch.float64
        gaps_n = self.K - 1
        avail = self.hi - self.lo
        if gaps_n == 0:
            return torch.full((n, 1), 0.5 * (self.lo + self.hi), dtype=dtype, device=self.device)
        room = self.max_distance - self.min_distance
        limit = avail - gaps_n * self.min_distance
        extras = torch.rand((n, gaps_n), dtype=dtype, device=self.device, generator=self.gen) * room
        scale = (limit / extras.sum(dim=1).clamp(min=1e-12)).clamp(max=1.0)
        gaps = extras * scale.unsqueeze(-1) + self.min_distance
        remaining = avail - gaps.sum(dim=1)
        offset = self.lo + 0.5 * remaining.unsqueeze(-1)
        return torch.cat([offset, offset + torch.cumsum(gaps, dim=1)], dim=1)


class CKM1DVecEnv:
    """Vectorised env: ``reset()`` then ``step(actions)``.

    ``actions``: (num_envs, 2) float32, PA_1 and PA_2 in bar.
    ``obs``: (num_envs, 2K) float32 = [x_1..x_K, R_1..R_K] (dimensionless),
    written in place by the step's graph.
    """

    def __init__(self, num_envs: int = 1024, num_bubbles: int = 4, R0_um: float = 60.0,
                 acoustic_field: str = "SW_N", freqs_khz=(25.0, 50.0), ref_freq_khz: float = 25.0,
                 time_step_length: float = 5.0, episode_length: int = 128, seed: int = 42,
                 position_tolerance: float = 0.01, dnorm: float = 0.2, reward_exp: float = 0.5,
                 rewards_weights=(1.0, 0.0), positive_terminal_reward: float = 10.0,
                 negative_terminal_reward: float = -10.0, max_steps: int = 1_000_000,
                 solver_spec: Optional[SolverSpec] = None, device: int = 0):
        import torch
        self.num_envs, self.K = int(num_envs), int(num_bubbles)
        self.time_step_length = float(time_step_length)
        self.episode_length = int(episode_length)
        self.position_tolerance = position_tolerance
        self.r_dnorm = 1.0 / dnorm
        self.reward_exp = reward_exp
        self.weights = rewards_weights
        self.pos_reward, self.neg_reward = positive_terminal_reward, negative_terminal_reward
        self.device = device
        self.tdev = torch.device("cuda", device)
        self.scenes = SceneGenerator(self.K, seed=seed, device=self.tdev)
        nk = len(freqs_khz)
        # physics: one uniform-K ensemble, initial PA (1, 0) bar as in the reference env defaults
        sc = scenes.Scene(K=np.full(self.num_envs, self.K, np.int32),
                          R0=[np.full(self.K, R0_um)] * self.num_envs,
                          PA=np.tile(np.array([1.0] + [0.0] * (nk - 1))[:, None], (1, self.num_envs)),
                          FR=np.tile(np.asarray(freqs_khz, dtype=np.float64)[:, None], (1, self.num_envs)),
                          PS=np.zeros((nk, self.num_envs)),
                          X0=[np.linspace(-0.4, 0.4, self.K)] * self.num_envs,
                          t_end=np.full(self.num_envs, self.time_step_length), ac=acoustic_field)
        self.ens = Ensemble.from_scene(sc, solver_spec=solver_spec, device=device)
        self.ens.to_device()
        d = self.ens.dev
        self.actions = torch.zeros((self.num_envs, nk), dtype=torch.float32, device=self.tdev)
        self.obs = torch.zeros((self.num_envs, 2 * self.K), dtype=torch.float32, device=self.tdev)
        self.failed = torch.zeros(self.num_envs, dtype=torch.uint8, device=self.tdev)
        self.targets = torch.zeros((self.num_envs, self.K), dtype=torch.float32, device=self.tdev)
        self.algo_steps = torch.zeros(self.num_envs, dtype=torch.long, device=self.tdev)
        self.total_rewards = torch.zeros(self.num_envs, dtype=torch.float32, device=self.tdev)
        io = _lib.cbc_env_io()
        io.actions = self.actions.data_ptr()
        io.n_act = nk
        io.act_stride = nk
        io.act_scale = 1.0e5           # bar -> Pa (reference action scale, :316-322)
        io.obs = self.obs.data_ptr()
        io.failed = self.failed.data_ptr()
        io.K = self.K
        io.t_span = self.time_step_length
        io.h0 = 1e-6                   # advance_time resets the step to 1e-6 (:816-826)
        self._io = io
        wl = make_work_list(self.ens.host["K"], np.full(self.num_envs, self.time_step_length))
        self._w, self._keep = self.ens.work(wl)
        self._spec, self._e = self.ens.spec(), self.ens.abi()
        self.ctx = _lib.default_context(device)
        h = _lib.P()
        self.ctx.check(_lib.lib().cbc_env_plan_create(self.ctx.handle, ctypes.byref(self._spec),
                                                      ctypes.byref(self._e), ctypes.byref(self._w),
                                                      int(max_steps), ctypes.byref(io), ctypes.byref(h)))
        self.plan = h.value
        # bubble rows of each env, for resets by index
        self._rows = torch.as_tensor(self.ens.host["bubble_offset"], device=self.tdev).unsqueeze(1) + \
            torch.arange(self.K, device=self.tdev).unsqueeze(0)

    # ---- resets ----
    def _write_scene(self, env_ids):
        import torch
        n = env_ids.numel()
        pos = self.scenes.positions(n)
        tgt = self.scenes.positions(n)
        st = self.ens.dev["state"]
        rows = self._rows[env_ids].reshape(-1)
        fresh = torch.zeros((rows.numel(), 4), dtype=torch.float64, device=self.tdev)
        fresh[:, 0] = 1.0
        fresh[:, 1] = pos.reshape(-1)
        st.index_copy_(0, rows, fresh)
        self.targets.index_copy_(0, env_ids, tgt.to(torch.float32))
        self.obs[env_ids, :self.K] = pos.to(torch.float32)
        self.obs[env_ids, self.K:] = 1.0
        self.algo_steps[env_ids] = 0
        self.total_rewards[env_ids] = 0.0

    def reset(self) -> Tuple[object, Dict]:
        import torch
        self._write_scene(torch.arange(self.num_envs, device=self.tdev))
        return self.obs, {}

    # ---- step ----
    def step_physics(self, stream=None) -> None:
        """Action -> control parameters, integrate, observation (one graph launch)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.ctx.check(_lib.lib().cbc_plan_launch(self.plan, ctypes.c_void_p(st.cuda_stream)))

    def step(self, actions=None):
        import torch
        if actions is not None:
            self.actions.copy_(actions)
        self.step_physics()
        x = self.obs[:, :self.K]
        failure = self.failed.bool()
        td = (self.targets - x).abs()
        success = torch.all(td <= self.position_tolerance, dim=1)
        td = td.masked_fill(td < self.position_tolerance, 0.0)
        dist = (td * self.r_dnorm).clamp(min=0.0).pow(self.reward_exp).mean(dim=1)
        intensity = self.actions.pow(2.0).sum(dim=1).sqrt()
        rewards = (-self.weights[0] * dist - self.weights[1] * intensity + self.neg_reward * failure.float()
                   + self.pos_reward * success.float())
        self.total_rewards += rewards
        self.algo_steps += 1
        terminated = failure | success
        time_outs = self.algo_steps >= self.episode_length
        done = torch.nonzero(terminated | time_outs).flatten()
        info = {}
        if done.numel() > 0:
            info = {"final_observation": self.obs[done].clone(), "dones": done,
                    "episode_return": self.total_rewards[done].clone(),
                    "episode_length": self.algo_steps[done].clone()}
            self._write_scene(done)
        return self.obs, rewards, terminated, time_outs, info

    def close(self) -> None:
        if getattr(self, "plan", None):
            _lib.lib().cbc_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
