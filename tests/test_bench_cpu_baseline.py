"""bench.py's CPU baseline (the oracle on all host cores, one system per
worker at a time) on a tiny bounded sample."""
import numpy as np


def test_cpu_baseline_small_sample():
    import bench
    from cbc_b200 import scenes
    sc = scenes.mixed_k(ns=32, seed=1)
    r = bench.cpu_baseline(sc, seconds=0.2, nthreads=2, step_cap=500)
    assert r["kind"] == "port" and r["cores"] == 2 and r["unit"] == bench.UNIT
    assert np.isfinite(r["value"]) and r["value"] > 0.0
    assert "systems drawn at random" in r["sample"] and "500-step cap" in r["sample"]
