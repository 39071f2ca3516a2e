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
