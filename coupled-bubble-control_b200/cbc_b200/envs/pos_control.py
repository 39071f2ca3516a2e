"""GPU-resident vectorised bubble position-control environment.

B200 counterpart of the reference's ``PosNBC1D``
(``coupledbubble_control/envs/bubble_1D_pos_control.py``): N coupled bubbles
per environment, the acoustic amplitudes (PA_1, PA_2) as the action, bubble
positions and radii as the observation, target positions, reward and
termination as in the reference (``get_rewards`` :792-813,
``check_termination`` :772-789, ``advance_time`` :816-826,
``final_termination`` :830-853), and random scene resets
(``SceneGenerator._random_uniform_position_1D`` :176-234, ``reset_envs``
:583-614).

One ``step`` is one CUDA-graph launch (``cbc_env_plan_create``): action ->
control parameters and time reset (prologue kernel), the batched integration
of ``time_step_length`` periods for every env, and one epilogue kernel that
writes the float32 observation straight into ``self.obs``, computes reward
and termination, and resets the envs that finished (new positions and
targets drawn on the device).  No torch op and no host synchronisation is
part of a step; the state stays on the device.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Tuple

import numpy as np

from .. import _lib, scenes
from ..ensemble import Ensemble, make_work_list
from ..models import SolverSpec

_M64 = (1 << 64) - 1


def _splitmix64(z: np.ndarray) -> np.ndarray:
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


class SceneGenerator:
    """Random chains of K bubbles inside [domain_min + margin, domain_max -
    margin]: K - 1 gaps of min_distance plus uniform extras up to
    max_distance - min_distance, scaled down to fit, centred (reference
    SceneGenerator, envs/bubble_1D_pos_control.py:46-249, 'random'
    positions, 'center' alignment).  The uniform draws are a counter-based
    hash (SplitMix64) of (seed, env, reset count, stream, draw), so the
    device epilogue (csrc/vecenv.cu) and this host restatement produce the
    same scenes."""

    def __init__(self, num_bubbles: int, min_distance: float = 0.05, max_distance: float = 0.9,
                 margin: float = 0.05, domain_min: float = -0.5, domain_max: float = 0.5, seed: int = 42):
        self.K = int(num_bubbles)
        self.min_distance, self.max_distance = float(min_distance), float(max_distance)
        self.lo, self.hi = domain_min + margin, domain_max - margin
        self.seed = int(seed) & _M64
        if (self.K - 1) * min_distance > self.hi - self.lo:
            raise ValueError(f"Cannot fit: the scene needs {(self.K - 1) * min_distance:.2f}, "
                             f"domain is {self.hi - self.lo:.2f}")

    def uniform(self, env: np.ndarray, count: np.ndarray, which: int, j: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            key = (np.uint64(self.seed) ^ (env.astype(np.uint64) * np.uint64(0xD1B54A32D192ED03))
                   ^ (count.astype(np.uint64) * np.uint64(0xABC98388FB8FAC03))
                   ^ np.uint64(((which * 64 + j) * 0x8CB92BA72F3D8DD7) & _M64))
            return (_splitmix64(key) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def positions(self, env, count, which: int = 0) -> np.ndarray:
        """(n, K) positions for envs `env` at their reset counts `count`
        (which = 0: bubble positions, 1: targets)."""
        env = np.atleast_1d(np.asarray(env, np.int64))
        count = np.broadcast_to(np.asarray(count, np.int64), env.shape)
        n, K = env.size, self.K
        if K == 1:
            return np.full((n, 1), 0.5 * (self.lo + self.hi))
        avail = self.hi - self.lo
        room = self.max_distance - self.min_distance
        limit = avail - (K - 1) * self.min_distance
        with np.errstate(over="ignore"):
            ext = np.stack([self.uniform(env, count, which, j) * room for j in range(K - 1)], 1)
        ssum = np.zeros(n)
        for j in range(K - 1):
            ssum = ssum + ext[:, j]
        sc = np.minimum(limit / np.maximum(ssum, 1e-12), 1.0)
        gsum = np.zeros(n)
        gaps = np.empty_like(ext)
        for j in range(K - 1):
            gaps[:, j] = ext[:, j] * sc + self.min_distance
            gsum = gsum + gaps[:, j]
        out = np.empty((n, K))
        out[:, 0] = self.lo + 0.5 * (avail - gsum)
        for j in range(K - 1):
            out[:, j + 1] = out[:, j] + gaps[:, j]
        return out


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
                 solver_spec: Optional[SolverSpec] = None, device: int = 0, envs_per_warp: int = 0):
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
        self.scenes = SceneGenerator(self.K, seed=seed)
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
        n = self.num_envs
        f32 = torch.float32
        z = lambda shape, dt: torch.zeros(shape, dtype=dt, device=self.tdev)   # noqa: E731
        self.actions = z((n, nk), f32)
        self.obs = z((n, 2 * self.K), f32)
        self.failed = z(n, torch.uint8)
        self.targets = z((n, self.K), f32)
        self.rewards = z(n, f32)
        self.terminated = z(n, torch.uint8)
        self.time_outs = z(n, torch.uint8)
        self.done = z(n, torch.uint8)
        self.algo_steps = z(n, torch.int32)
        self.total_rewards = z(n, f32)
        self.final_obs = z((n, 2 * self.K), f32)
        self.episode_return = z(n, f32)
        self.episode_len = z(n, torch.int32)
        self.reset_count = z(n, torch.int64)
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
        for name in ("targets", "rewards", "terminated", "time_outs", "done", "algo_steps", "total_rewards",
                     "final_obs", "episode_return", "episode_len", "reset_count"):
            setattr(io, name, getattr(self, name).data_ptr())
        io.position_tolerance = position_tolerance
        io.r_dnorm = self.r_dnorm
        io.reward_exp = reward_exp
        io.w_dist, io.w_intensity = float(rewards_weights[0]), float(rewards_weights[1])
        io.pos_reward, io.neg_reward = positive_terminal_reward, negative_terminal_reward
        g = self.scenes
        io.min_distance, io.max_distance, io.domain_lo, io.domain_hi = g.min_distance, g.max_distance, g.lo, g.hi
        io.episode_length = self.episode_length
        io.seed = g.seed
        self._io = io
        wl = make_work_list(self.ens.host["K"], np.full(self.num_envs, self.time_step_length))
        # envs per warp: 0 packs floor(32 / K).  Fewer leave lanes idle and
        # free each env from the Richardson sweeps of its warp-mates, but the
        # extra warps share the SMs' issue slots: 1024 envs of K = 4 stepped
        # in 68 ms packed, 77 ms at 2 and 87 ms at 1 env per warp
        if envs_per_warp > 0:
            wl.slots = np.full(wl.bucket_K.size, min(int(envs_per_warp), 32 // self.K), np.int32)
        self._w, self._keep = self.ens.work(wl)
        self._spec, self._e = self.ens.spec(), self.ens.abi()
        self.ctx = _lib.default_context(device)
        h = _lib.P()
        self.ctx.check(_lib.lib().cbc_env_plan_create(self.ctx.handle, ctypes.byref(self._spec),
                                                      ctypes.byref(self._e), ctypes.byref(self._w),
                                                      int(max_steps), ctypes.byref(io), ctypes.byref(h)))
        self.plan = h.value
        torch.cuda.synchronize(device)

    # ---- resets ----
    def reset(self) -> Tuple[object, Dict]:
        """New scenes for every env (device kernel, the same draws and
        formulas as the step's in-graph resets)."""
        import torch
        st = torch.cuda.current_stream(self.device)
        self.ctx.check(_lib.lib().cbc_env_reset(self.ctx.handle, ctypes.byref(self._e), ctypes.byref(self._io),
                                                None, ctypes.c_void_p(st.cuda_stream)))
        return self.obs, {}

    # ---- step ----
    def step_physics(self, stream=None) -> None:
        """One environment step for every env (one graph launch)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.ctx.check(_lib.lib().cbc_plan_launch(self.plan, ctypes.c_void_p(st.cuda_stream)))

    def step(self, actions=None):
        """Returns (obs, rewards, terminated, time_outs, info), all device
        tensors written by the step's graph.  info['done'] marks the envs
        that finished in this step and were reset; their last observation,
        return and length are in info['final_observation'],
        info['episode_return'] and info['episode_length'] (valid where done)."""
        if actions is not None:
            self.actions.copy_(actions)
        self.step_physics()
        info = {"done": self.done, "final_observation": self.final_obs, "episode_return": self.episode_return,
                "episode_length": self.episode_len}
        return self.obs, self.rewards, self.terminated, self.time_outs, info

    def close(self) -> None:
        if getattr(self, "plan", None):
            _lib.lib().cbc_plan_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
