"""Host-side work-list construction of the batched solve (no GPU)."""
import numpy as np

from cbc_b200.ensemble import make_work_list


def test_latency_lane_work_list():
    """Latency lanes take the longest serial chains, keep every system exactly
    once and stay inside the SM budget (4 warps of 32 // K systems per SM)."""
    from cbc_b200.ensemble import with_latency_lane
    rng = np.random.default_rng(3)
    K = rng.choice([2, 3, 4, 8], size=2000)
    work = rng.uniform(1.0, 10.0, size=2000)
    work[7] = 1e4                      # one dominant chain
    wl = with_latency_lane(make_work_list(K, work), K, work, fraction=0.02, max_sms=5)
    assert sorted(wl.order.tolist()) == list(range(2000))
    ex = wl.exclusive
    assert ex is not None and ex.shape == wl.bucket_K.shape and 1 <= ex.sum() <= 5
    lanes = [b for b in range(ex.size) if ex[b] > 0]
    in_lane = np.concatenate([wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]] for b in lanes])
    assert 7 in in_lane.tolist()
    for b in lanes:
        k = int(wl.bucket_K[b])
        seg = wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]]
        assert np.all(K[seg] == k) and seg.size <= ex[b] * 4 * (32 // k)
    assert np.all(wl.share[lanes] == 0)


def test_adaptive_replanning_host_logic():
    """AdaptivePlan's re-planning step: rates from observed progress, the
    systems that would end last go to latency lanes (longest first, inside
    the SM budget), every active system appears exactly once, finished ones
    not at all."""
    from cbc_b200.ensemble import adaptive_work_list, alone_latency
    rng = np.random.default_rng(5)
    n = 3000
    K = rng.choice([2, 3, 4, 6, 8], size=n)
    t_end = rng.uniform(5.0, 50.0, n)
    t0 = np.zeros(n)
    t = rng.uniform(0.0, 1.0, n)
    rate = rng.uniform(500, 3000, n)
    rate[:5] = 12000.0                     # five systems that step very slowly through time
    attempts = (rate * t).astype(np.int64)
    a0 = np.zeros(n, np.int64)
    active = np.ones(n, bool)
    active[100:200] = False                # finished
    wl, info = adaptive_work_list(K, t_end, t0, a0, t, attempts, active, sm_count=148, max_lane_sms=8)
    assert sorted(wl.order.tolist()) == sorted(np.nonzero(active)[0].tolist())
    assert info["lane_systems"] > 0 and 1 <= info["lane_sms"] <= 8
    lanes = [b for b in range(wl.bucket_K.size) if wl.exclusive[b] > 0]
    in_lane = set(np.concatenate([wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]] for b in lanes]).tolist())
    # long serial chains: remaining attempts x their alone latency well past the bulk time
    slow = [i for i in range(5) if (t_end[i] - t[i]) * 12000.0 * alone_latency(K[i])[0] * 1e-6 > 2.0]
    assert set(slow) <= in_lane
    # with no observations yet the fallback rate still yields a complete list
    # inside the default lane budget of 32 SMs
    wl2, info2 = adaptive_work_list(K, np.full(n, 0.01), t0, a0, t0, a0, active, sm_count=148)
    assert sorted(wl2.order.tolist()) == sorted(np.nonzero(active)[0].tolist()) and info2["lane_sms"] <= 32


def test_solo_lanes_keep_every_system_once():
    """Solo lanes (one system per warp) for the longest chains: every active
    system appears exactly once in the work list, solo buckets hold one
    system per warp and four per exclusive SM."""
    from cbc_b200.ensemble import adaptive_work_list
    rng = np.random.default_rng(5)
    n = 3000
    K = rng.choice([2, 3, 4, 8], size=n)
    t_end = rng.uniform(5.0, 50.0, size=n)
    t0 = np.zeros(n)
    a0 = np.zeros(n, np.int64)
    t = rng.uniform(0.0, 1.0, size=n)
    attempts = (t * rng.uniform(500, 20000, size=n)).astype(np.int64) + 300
    active = np.ones(n, bool)
    for solo in (0, 3, 8):
        wl, info = adaptive_work_list(K, t_end, t0, a0, t, attempts, active, 148, max_lane_sms=16, solo=solo)
        assert sorted(wl.order.tolist()) == list(range(n))
        assert info["solo_systems"] == min(solo, info["lane_systems"])
        if solo and info["solo_systems"]:
            solo_b = [b for b in range(wl.bucket_K.size) if wl.slots is not None and wl.slots[b] == 1]
            assert solo_b
            for b in solo_b:
                seg = wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]]
                assert wl.exclusive[b] == (seg.size + 3) // 4 and np.all(K[seg] == wl.bucket_K[b])


def test_lane_threshold_monotone():
    """The latency-lane criterion multiplies a system's serial time by
    `load_factor`: a larger factor never puts fewer systems into lanes, and
    the chosen systems are the longest chains."""
    from cbc_b200.ensemble import adaptive_work_list, alone_latency
    rng = np.random.default_rng(11)
    n = 4000
    K = rng.choice([2, 3, 4, 6, 8], size=n)
    t_end = rng.uniform(5.0, 50.0, n)
    t0 = np.zeros(n)
    t = rng.uniform(0.0, 2.0, n)
    rate = rng.uniform(500, 3000, n)
    rate[:40] = rng.uniform(8000, 14000, 40)
    attempts = (rate * t).astype(np.int64)
    a0 = np.zeros(n, np.int64)
    active = np.ones(n, bool)
    counts = []
    for lf in (0.8, 1.0, 1.2, 1.35, 1.6, 2.0):
        wl, info = adaptive_work_list(K, t_end, t0, a0, t, attempts, active, sm_count=148, max_lane_sms=32,
                                      load_factor=lf)
        assert sorted(wl.order.tolist()) == list(range(n))
        counts.append(info["lane_systems"])
        if info["lane_systems"]:
            lanes = [b for b in range(wl.bucket_K.size) if wl.exclusive[b] > 0]
            in_lane = np.concatenate([wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]] for b in lanes])
            # systems with enough attempts to use their own rate: every lane
            # system's predicted serial time is at least that of those left out
            own = attempts >= 256
            serial = (t_end - t) * (attempts / np.maximum(t, 1e-12)) * alone_latency(K)
            out = np.setdiff1d(np.nonzero(own)[0], in_lane)
            lane_own = in_lane[own[in_lane]]
            if lane_own.size and out.size:
                assert serial[lane_own].min() >= serial[out].max() * 0.999
    assert counts == sorted(counts)
