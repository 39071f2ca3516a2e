"""Trajectory streaming: dense output of a solved ensemble -> pinned host
buffers -> sharded files.

Counterpart of the reference's ``TrajectorBuffer`` (``envs/common/
trajectory_buffer.py:95-226``), which copies every env's dense output to the
host with a per-step ``.cpu()`` and a Python loop over envs, then writes a
sharded zarr store.  Here the samples stay in the ensemble's sample-major
device arrays (``dense_time`` (ndo, ns), ``dense_state`` (ndo, nb, 4)) until
they are streamed shard by shard: each shard (a contiguous range of systems,
hence of bubble rows) is copied device -> pinned host on a side stream into
one of two staging buffers while the host writes the previous shard to disk,
so copies and file writes overlap.  Shards are ``.npz`` files (zarr is not a
dependency of this package) holding K, the bubble offsets relative to the
shard, dense_index, dense_time and dense_state of their systems, plus a
``manifest.json``.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List

import numpy as np


class TrajectoryWriter:
    def __init__(self, ens, out_dir: str, shard_systems: int = 4096):
        if ens.ndo <= 0:
            raise ValueError("the ensemble has no dense output (ndo = 0)")
        self.ens = ens
        self.out_dir = out_dir
        self.shard_systems = int(shard_systems)

    def _shards(self):
        ns = self.ens.ns
        for s0 in range(0, ns, self.shard_systems):
            yield s0, min(ns, s0 + self.shard_systems)

    def write(self) -> List[str]:
        """Streams every shard; returns the shard paths (after the manifest
        is written).  Call after the solve that produced the samples."""
        import torch
        ens = self.ens
        d, h = ens.dev, ens.host
        os.makedirs(self.out_dir, exist_ok=True)
        boff = h["bubble_offset"]
        K = h["K"]
        side = torch.cuda.Stream(device=ens.device)
        side.wait_stream(torch.cuda.current_stream(ens.device))   # after the solve
        nmax = self.shard_systems
        bmax = int(max(int(boff[e - 1] + K[e - 1] - boff[s]) for s, e in self._shards()))
        stage = [{"t": torch.empty((ens.ndo, nmax), dtype=torch.float64).pin_memory(),
                  "x": torch.empty((ens.ndo, bmax, 4), dtype=torch.float64).pin_memory(),
                  "i": torch.empty(nmax, dtype=torch.int32).pin_memory(),
                  "ev": torch.cuda.Event()} for _ in range(2)]
        paths: List[str] = []
        pending = None

        def flush(item):
            buf, s0, s1, b0, b1, path = item
            buf["ev"].synchronize()
            np.savez(path, K=K[s0:s1], bubble_offset=boff[s0:s1] - b0,
                     dense_index=buf["i"][:s1 - s0].numpy().copy(),
                     dense_time=buf["t"][:, :s1 - s0].numpy().copy(),
                     dense_state=buf["x"][:, :b1 - b0].numpy().copy())
            paths.append(path)

        for n, (s0, s1) in enumerate(self._shards()):
            b0, b1 = int(boff[s0]), int(boff[s1 - 1] + K[s1 - 1])
            buf = stage[n & 1]
            with torch.cuda.stream(side):
                buf["t"][:, :s1 - s0].copy_(d["dense_time"][:, s0:s1], non_blocking=True)
                buf["x"][:, :b1 - b0].copy_(d["dense_state"][:, b0:b1], non_blocking=True)
                buf["i"][:s1 - s0].copy_(d["dense_index"][s0:s1], non_blocking=True)
                buf["ev"].record(side)
            if pending is not None:
                flush(pending)                # the previous shard, while this one copies
            pending = (buf, s0, s1, b0, b1, os.path.join(self.out_dir, f"shard_{n:05d}.npz"))
        if pending is not None:
            flush(pending)
        manifest: Dict[str, object] = {"ns": ens.ns, "nb": ens.nb, "ndo": ens.ndo,
                                       "shard_systems": self.shard_systems,
                                       "shards": [os.path.basename(p) for p in paths]}
        with open(os.path.join(self.out_dir, "manifest.json"), "w") as f:
            json.dump(manifest, f)
        return paths


def read_trajectories(out_dir: str) -> Dict[str, np.ndarray]:
    """Reassembles the sharded dense output (dense_index, dense_time,
    dense_state in the ensemble's layout)."""
    with open(os.path.join(out_dir, "manifest.json")) as f:
        man = json.load(f)
    idx, t, x = [], [], []
    for name in man["shards"]:
        z = np.load(os.path.join(out_dir, name))
        idx.append(z["dense_index"])
        t.append(z["dense_time"])
        x.append(z["dense_state"])
    return {"dense_index": np.concatenate(idx), "dense_time": np.concatenate(t, axis=1),
            "dense_state": np.concatenate(x, axis=1)}
