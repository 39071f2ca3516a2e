"""PPO rollout collection with the env step captured in a CUDA graph
(cbc_b200.rollout): a graphed rollout's transitions equal an eager replay of
its recorded actions on a twin env, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graphed_rollout_equals_eager_replay(cuda):
    import torch
    from cbc_b200.envs import CKM1DVecEnv
    from cbc_b200.rollout import ActorCritic, GraphedRollout
    n, K, T = 32, 4, 6
    torch.manual_seed(0)
    kw = dict(num_envs=n, num_bubbles=K, time_step_length=0.02, episode_length=3, seed=5, position_tolerance=0.05)
    env = CKM1DVecEnv(**kw)
    env.reset()
    pol = ActorCritic(2 * K, 2).cuda()
    ro = GraphedRollout(env, pol, T)
    ro.capture()                       # warm-up advanced env once: replay the twin from that point
    twin = CKM1DVecEnv(**kw)
    twin.reset()
    twin.step(ro.buf["actions"][0].clamp(0.0, 1.5))
    out = ro.collect()
    torch.cuda.synchronize()
    for t in range(T):
        assert torch.equal(twin.obs, out["obs"][t])
        twin.step(out["actions"][t].clamp(0.0, 1.5))
        torch.cuda.synchronize()
        assert torch.equal(twin.rewards, out["raw_rewards"][t])
        assert torch.equal(twin.done.float(), out["dones"][t])
    assert torch.isfinite(out["advantages"]).all() and out["dones"].sum() > 0
    env.close()
    twin.close()
