"""Trajectory streaming (cbc_b200.trajectory): the dense output of a solved
ensemble, streamed shard by shard through pinned buffers to files and read
back, equals the device arrays exactly."""
import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.ensemble import Ensemble
from cbc_b200.trajectory import TrajectoryWriter, read_trajectories


def test_rejects_ensembles_without_dense_output():
    ens = Ensemble.from_scene(scenes.mixed_k(ns=8, span=(0.1, 0.2), seed=80))
    with pytest.raises(ValueError):
        TrajectoryWriter(ens, "unused")


@pytest.mark.gpu
def test_stream_round_trip(cuda, tmp_path):
    import torch
    sc = scenes.mixed_k(ns=700, span=(0.1, 0.3), seed=81)
    sc.ndo = 12
    ens = Ensemble.from_scene(sc).to_device()
    ens.solve(200_000)
    paths = TrajectoryWriter(ens, str(tmp_path), shard_systems=128).write()
    torch.cuda.synchronize()
    assert len(paths) == 6
    got = read_trajectories(str(tmp_path))
    h = ens.to_host()
    for k in ("dense_index", "dense_time", "dense_state"):
        assert np.array_equal(got[k], h[k]), k
    assert int(h["dense_index"].min()) >= 1
