"""Continuous batching: a request's result is the same alone and in a mix
of concurrently served requests (bit for bit: every chunk resumes exactly
where the previous one stopped), and every request completes."""
import numpy as np
import pytest

from cbc_b200.serving import Request, SolveServer, latency_stats

pytestmark = pytest.mark.gpu


def make_requests(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        K = int(rng.choice([2, 4, 8]))
        R0 = rng.uniform(2, 8, K)
        x = np.sort(rng.uniform(-0.25, 0.25 - (K - 1) * 0.003, K)) + np.arange(K) * 0.003
        out.append(Request(rid=i, K=K, R0=R0, PA=rng.uniform(0, 1.5, 2), PS=rng.uniform(0, 2, 2), X0=x,
                           span=float(rng.uniform(0.05, 0.3))))
    return out


def run(reqs, slots, chunk):
    srv = SolveServer(slots, chunk_steps=chunk, keep_results=True)
    pending = list(reqs)
    it = 0
    while pending or not srv.idle():
        # staggered arrivals: a few new requests per loop iteration
        for _ in range(3):
            if pending:
                r = pending.pop(0)
                r.arrival = srv.now()
                srv.submit(r)
        srv.step()
        it += 1
        assert it < 100000
    return {r.rid: r for r in srv.completed}


def test_alone_equals_in_mix(cuda):
    reqs = make_requests(60, seed=4)
    mix = run(make_requests(60, seed=4), {2: 16, 4: 8, 8: 8}, chunk=97)
    assert len(mix) == 60
    for r in reqs[:6]:
        alone = run([r], {r.K: 1}, chunk=1000000)[r.rid]
        a, b = alone.result, mix[r.rid].result
        assert np.array_equal(a["state"], b["state"]) and a["t"] == b["t"] and a["status"] == b["status"]
        assert a["steps"] == b["steps"] and a["h"] == b["h"]
    stats = latency_stats(list(mix.values()))
    assert stats["completed"] == 60 and stats["p99_ms"] >= stats["p50_ms"] > 0


def test_admission_by_memory_and_fifo(cuda):
    """Pools sized for two K = 8 requests: the third waits for memory (and a
    later K = 2 request does not overtake it); everything completes."""
    from cbc_b200.serving import SolveServer as S
    srv = S(max_systems=8, memory_bytes=0, slice_ms=1.0, keep_results=False)
    srv.rows = type(srv.rows)(16)                       # room for 16 bubble rows
    srv.coup = type(srv.coup)(2 * 3 * 64)               # and two K = 8 coupling blocks
    reqs = make_requests(40, seed=9)
    k8 = [r for r in reqs if r.K == 8][:3]
    k2 = [r for r in reqs if r.K == 2][:1]
    for r in k8 + k2:
        r.arrival = 0.0
        srv.submit(r)
    srv._admit()
    assert len(srv.busy) == 2 and len(srv.queue) == 2 and srv.queue[0] is k8[2]
    it = 0
    while not srv.idle():
        srv.step()
        it += 1
        assert it < 100000
    assert {r.rid for r in srv.completed} == {r.rid for r in k8 + k2}
    assert srv.rows.used == 0 and srv.coup.used == 0 and len(srv.free_slots) == 8
