"""The multi-rank (N > 1) reduction of bench.py on CPU with gloo, world size 2:
max over ranks of the time, sum of the work, distinct per-rank ensembles."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, work = bench.job_totals(100.0 + 50.0 * rank, 10.0 * (rank + 1), dist, "cpu")
    q.put((rank, ms, work, bench.rank_seed(rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_job_totals_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    for rank, ms, work, seed in res:
        assert ms == 150.0 and work == 30.0
    assert res[0][3] != res[1][3]


def test_job_totals_single():
    import bench
    assert bench.job_totals(5.0, 7.0) == (5.0, 7.0)
