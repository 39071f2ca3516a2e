"""The reference arm of bench.py (`--impl reference`): one JSON line with the
contract's keys, the CPU baseline describing the run and a zero-copy e2e,
on a tiny workload with short samples (the oracle on the host cores)."""
import argparse
import json

import bench


def test_reference_arm_line(monkeypatch, capsys):
    real = bench.cpu_baseline
    monkeypatch.setattr(bench, "cpu_baseline",
                        lambda scene, seconds=12.0, seed=99: real(scene, seconds=0.05, nthreads=2, seed=seed,
                                                                  step_cap=300))
    args = argparse.Namespace(ns=32, steps=2, warmup=3, gpus=1, only_k=0, max_steps=bench.MAX_STEPS,
                              lin_solver="richardson", schedule="adaptive")
    bench.run_reference(args)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["value"] > 0.0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 2
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "mixed_k_32"
