"""The seeded synthetic workloads: bubble positions sorted with a minimum gap
of 20 max(R0) / lambda_1 inside the stated range, parameter ranges, the
mixed-K weights and spans, and reproducibility by seed."""
import numpy as np

from cbc_b200 import scenes


def _check_positions(sc, lo, hi):
    for s in range(sc.ns):
        x = np.asarray(sc.X0[s])
        gmin = 20.0 * np.max(sc.R0[s]) * 1e-6 / scenes.LAMBDA1
        assert np.all(np.diff(x) >= gmin * (1 - 1e-12))
        assert x[0] >= lo and x[-1] <= hi


def test_mixed_k_workload():
    sc = scenes.mixed_k(ns=20000, seed=1)
    assert set(np.unique(sc.K).tolist()) == {2, 3, 4, 6, 8}
    frac = np.array([np.mean(sc.K == k) for k in (2, 3, 4, 6, 8)])
    assert np.all(np.abs(frac - np.array([0.4, 0.2, 0.2, 0.1, 0.1])) < 0.015)
    assert sc.t_end.min() >= 5.0 and sc.t_end.max() <= 50.0
    assert all(np.all((np.asarray(r) >= 2.0) & (np.asarray(r) <= 8.0)) for r in sc.R0)
    assert np.all((sc.PA >= 0.0) & (sc.PA <= 1.5))
    assert np.all((sc.PS >= 0.0) & (sc.PS < 2.0))
    _check_positions(scenes.subset(sc, np.arange(2000)), -0.25, 0.25)
    again = scenes.mixed_k(ns=20000, seed=1)
    assert np.array_equal(again.K, sc.K) and np.array_equal(again.t_end, sc.t_end)


def test_plain_and_large_k_workloads():
    p = scenes.plain_study(ns=256, periods=10.0, samples_per_period=32, seed=0)
    assert np.all(p.K == 2) and p.ndo == 321 and np.all(p.t_end == 10.0)
    _check_positions(p, -0.25, 0.25)
    lk = scenes.large_k(ns=8, K=32, periods=200.0, samples_per_period=64, seed=4)
    assert np.all(lk.K == 32) and lk.ndo == 12801
    _check_positions(lk, -0.5, 0.5)


def test_env_scene_generator_draws():
    """Host restatement of the env's device scene generator: chains inside
    the domain with gaps >= min_distance, different per env and per reset."""
    from cbc_b200.envs import SceneGenerator
    g = SceneGenerator(4, seed=5)
    p = g.positions(np.arange(200), 0, 0)
    assert p.shape == (200, 4)
    gaps = np.diff(p, axis=1)
    assert np.all(gaps >= g.min_distance - 1e-12) and np.all(p >= g.lo - 1e-12) and np.all(p <= g.hi + 1e-12)
    assert not np.array_equal(p, g.positions(np.arange(200), 1, 0))
    assert not np.array_equal(p, g.positions(np.arange(200), 0, 1))
    assert np.array_equal(p, SceneGenerator(4, seed=5).positions(np.arange(200), 0, 0))
