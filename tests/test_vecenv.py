"""Vec-env step on the GPU (one graph launch: action -> control parameters,
time reset, batched integration, then one epilogue kernel for the float32
observation, reward, termination and the resets of finished envs) against
the oracle, a torch restatement of the reference's reward and termination
(envs/bubble_1D_pos_control.py:772-813) and the host restatement of the
scene generator."""
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
    done = env.done.cpu().numpy().astype(bool)
    seen = np.where(done[:, None], env.final_obs.cpu().numpy(), env.obs.cpu().numpy())
    assert np.array_equal(seen[:, :4], x) and np.array_equal(seen[:, 4:], R)
    assert np.array_equal(env.failed.cpu().numpy(), (ref["status_flags"] != 1).astype(np.uint8))
    after = env.ens.to_host()["state"].reshape(48, 4, 4)
    want = np.transpose(ref["actual_state"], (1, 2, 0))
    assert np.array_equal(after[~done], want[~done])
    env.close()


def test_envs_per_warp_bit_identical(cuda):
    """One env per warp (idle lanes, no shared Richardson loop) gives the
    same step results as the packed default."""
    import torch
    from cbc_b200.envs import CKM1DVecEnv
    out = []
    for epw in (0, 1):
        env = CKM1DVecEnv(num_envs=40, num_bubbles=4, time_step_length=0.05, episode_length=2, seed=9,
                          envs_per_warp=epw)
        env.reset()
        gen = torch.Generator(device="cuda").manual_seed(4)
        res = []
        for _ in range(3):
            obs, rew, term, trunc, info = env.step(torch.rand((40, 2), device="cuda", generator=gen) * 1.5)
            torch.cuda.synchronize()
            res.append((obs.cpu().numpy().copy(), rew.cpu().numpy().copy(), env.ens.to_host()["state"].copy()))
        env.close()
        out.append(res)
    for a, b in zip(*out):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def _torch_reward(x, targets, failed, actions, tol=0.01, dnorm=0.2, exp=0.5, w=(1.0, 0.0), pos=10.0, neg=-10.0):
    """The reference's reward and termination (get_rewards :792-813,
    check_termination :772-789) in torch float32."""
    import torch
    td = (targets - x).abs()
    success = torch.all(td <= tol, dim=1)
    td = td.masked_fill(td < tol, 0.0)
    dist = (td * (1.0 / dnorm)).clamp(min=0.0).pow(exp).mean(dim=1)
    intensity = actions.pow(2.0).sum(dim=1).sqrt()
    reward = -w[0] * dist - w[1] * intensity + neg * failed.float() + pos * success.float()
    return reward, failed | success


def test_reward_termination_and_resets(cuda):
    import torch
    from cbc_b200.envs import CKM1DVecEnv, SceneGenerator
    n, K = 96, 4
    env = CKM1DVecEnv(num_envs=n, num_bubbles=K, time_step_length=0.03, episode_length=2, seed=11,
                      position_tolerance=0.05)
    env.reset()
    torch.cuda.synchronize()
    gen = SceneGenerator(K, seed=11)
    ids = np.arange(n)
    p0 = gen.positions(ids, 0, 0)
    assert np.array_equal(env.ens.to_host()["state"].reshape(n, K, 4)[:, :, 1], p0)
    assert np.array_equal(env.targets.cpu().numpy(), gen.positions(ids, 0, 1).astype(np.float32))
    assert np.array_equal(env.obs.cpu().numpy()[:, :K], p0.astype(np.float32))
    act = torch.rand((n, 2), device="cuda", generator=torch.Generator(device="cuda").manual_seed(3)) * 1.2
    for step in range(3):
        tgt = env.targets.clone()
        steps_before = env.algo_steps.clone()
        obs, rew, term, tout, info = env.step(act)
        torch.cuda.synchronize()
        done = info["done"].bool()
        x = torch.where(done[:, None], info["final_observation"], obs)[:, :K]
        r_ref, term_ref = _torch_reward(x, tgt, env.failed.bool(), act, tol=0.05)
        assert torch.allclose(rew, r_ref, rtol=1e-6, atol=1e-6)
        assert torch.equal(term.bool(), term_ref)
        assert torch.equal(tout.bool(), steps_before + 1 >= 2)
        assert torch.equal(done, term.bool() | tout.bool())
        d = done.cpu().numpy()
        if d.any():
            cnt = env.reset_count.cpu().numpy()
            assert np.all(cnt[d] >= 2)
            newpos = gen.positions(ids[d], cnt[d] - 1, 0)
            assert np.array_equal(obs.cpu().numpy()[d, :K], newpos.astype(np.float32))
            assert np.all(env.algo_steps.cpu().numpy()[d] == 0)
            assert np.array_equal(info["episode_length"].cpu().numpy()[d], (steps_before + 1).cpu().numpy()[d])
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
