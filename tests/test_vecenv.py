"""Vec-env step on the GPU (one graph launch: action -> control parameters,
time reset, batched integration, float32 observation) against the oracle."""
import numpy as np
import pytest

from cbc_b200.models import SolverSpec
from oracle import oracle

from _parity import ensemble_uniform_to_ref

pytestmark = pytest.mark.gpu


def test_env_step_matches_oracle(cuda):
    import torch
    from cbc_b200.envs import CKM1DVecEnv
    env = CKM1DVecEnv(num_envs=48, num_bubbles=4, time_step_length=0.05, seed=7)
    obs, _ = env.reset()
    torch.cuda.synchronize()
    before = env.ens.to_host()
    gen = torch.Generator(device="cuda").manual_seed(2)
    actions = torch.rand((48, 2), device="cuda", generator=gen) * 1.5
    env.actions.copy_(actions)
    env.step_physics()
    torch.cuda.synchronize()
    # oracle on the same state with the step's prologue applied on the host
    ref = ensemble_uniform_to_ref(before, 4, 2)
    a = actions.cpu().numpy().astype(np.float64)
    ref["control_params"][0:2, :] = (a * 1e5).T
    ref["actual_time"][:] = 0.0
    ref["time_end"][:] = 0.05
    ref["time_step"][:] = 1e-6
    ref["actual_event"][:] = -1.0
    ref["status_flags"][:] = 0
    spec = oracle.make_spec(48, 4, 4, 0, 2, "SW_N", SolverSpec())
    oracle.solve_ref_layout(spec, ref, 1_000_000)
    x = ref["actual_state"][1].astype(np.float32)
    R = ref["actual_state"][0].astype(np.float32)
    got = env.obs.cpu().numpy()
    assert np.array_equal(got[:, :4], x) and np.array_equal(got[:, 4:], R)
    assert np.array_equal(env.failed.cpu().numpy(), (ref["status_flags"] != 1).astype(np.uint8))
    after = env.ens.to_host()
    assert np.array_equal(after["state"].reshape(48, 4, 4), np.transpose(ref["actual_state"], (1, 2, 0)))
    env.close()


def test_env_episode_runs_and_resets(cuda):
    import torch
    from cbc_b200.envs import CKM1DVecEnv
    env = CKM1DVecEnv(num_envs=64, num_bubbles=4, time_step_length=0.05, episode_length=3, seed=1)
    obs, _ = env.reset()
    ptr = obs.data_ptr()
    for i in range(4):
        act = torch.full((64, 2), 0.5, device="cuda")
        obs, rew, term, tout, info = env.step(act)
        assert obs.data_ptr() == ptr            # observation is written in place (no copy)
        assert obs.dtype == torch.float32 and obs.shape == (64, 8)
        assert torch.isfinite(rew).all()
    assert int(env.algo_steps.max()) <= 3      # time-outs were reset
    env.close()
