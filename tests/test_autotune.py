"""The project-written autotuner (cbc_b200/autotune.py): search space,
selection rule and cache on the CPU; on the GPU, that every launch shape it
can pick gives bit-identical results and that a tuned ensemble solves to the
same answer as an untuned one."""
import numpy as np
import pytest

from cbc_b200 import autotune, scenes
from cbc_b200.autotune import DEFAULT, TuneConfig
from cbc_b200.ensemble import Ensemble, make_work_list

KEYS = ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters")


def test_candidates_cover_the_knobs():
    for K in (1, 2, 3, 4, 6, 8, 16, 32):
        c = autotune.candidates(K)
        assert c[0] == DEFAULT
        assert len(set(c)) == len(c)
        assert {x.threads for x in c} >= {128, 64}
        assert all(x.slots == 0 or 1 <= x.slots <= 32 // K for x in c)
        if K <= 8:
            assert {x.min_blocks for x in c} == {0, 1}
        else:
            assert {x.min_blocks for x in c} == {0}
    assert TuneConfig(128, 8, 0) in autotune.candidates(2)      # half-filled warps for K = 2


def test_choose_keeps_default_within_noise():
    a, b = DEFAULT, TuneConfig(64, 0, 1)
    assert autotune.choose({a: 100.0, b: 101.0}) == a
    assert autotune.choose({a: 100.0, b: 110.0}) == b
    assert autotune.choose({a: 100.0, b: 90.0}) == a
    assert autotune.choose({}) == DEFAULT


def test_tune_k_with_a_model_measurement():
    # a fake device where 64-thread blocks with the smaller register budget win
    def measure(cfg):
        return 1000.0 * (1.3 if (cfg.threads == 64 and cfg.min_blocks == 1) else 1.0) / (1 + (cfg.slots > 0))
    res = autotune.tune_k(4, measure)
    assert res["config"] == TuneConfig(64, 0, 1)
    assert abs(res["gain_vs_default"] - 1.3) < 1e-12
    assert len(res["rates"]) == len(autotune.candidates(4))


def test_cache_round_trip(tmp_path):
    p = str(tmp_path / "t.json")
    key = autotune.cache_key("NVIDIA B200", 100, 2, "lu", 8)
    autotune.save_cache({key: {"config": {"threads": 64, "slots": 2, "min_blocks": 1}, "rates": {},
                               "gain_vs_default": 1.1}}, p)
    t = autotune.load_cache(p)
    assert TuneConfig(**t[key]["config"]) == TuneConfig(64, 2, 1)
    assert autotune.load_cache(str(tmp_path / "missing.json")) == {}


def test_tuning_fills_work_list_arrays():
    sc = scenes.mixed_k(ns=200, span=(0.2, 0.3), seed=60)
    ens = Ensemble.from_scene(sc)
    wl = make_work_list(ens.host["K"], ens.host["t_end"])
    ens.tuning = {2: TuneConfig(64, 8, 1), 8: TuneConfig(32, 2, 0)}
    arr = ens._tuned_arrays(wl)
    for b, k in enumerate(wl.bucket_K):
        if k == 2:
            assert (arr["threads"][b], arr["slots"][b], arr["min_blocks"][b]) == (64, 8, 1)
        elif k == 8:
            assert (arr["threads"][b], arr["slots"][b], arr["min_blocks"][b]) == (32, 2, 0)
        else:
            assert (arr["threads"][b], arr["slots"][b], arr["min_blocks"][b]) == (128, 32 // k, 0)


def _compare(ha, hb):
    for k in KEYS:
        x, y = ha[k], hb[k]
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert np.all(same), f"{k}: {np.count_nonzero(~same)} mismatches"


@pytest.mark.gpu
@pytest.mark.parametrize("lin", ["richardson", "lu"])
def test_every_launch_shape_is_bit_identical(cuda, lin):
    import torch
    from cbc_b200.models import SolverSpec
    sc = scenes.mixed_k(ns=400, span=(0.2, 0.6), seed=61)
    spec = SolverSpec(lin_solver=lin)
    ref = Ensemble.from_scene(sc, solver_spec=spec).to_device()
    ref.solve(200_000)
    torch.cuda.synchronize()
    href = ref.to_host()
    for cfg in (TuneConfig(64, 0, 1), TuneConfig(32, 0, 0), TuneConfig(128, 1, 1), TuneConfig(96, 1, 0)):
        ens = Ensemble.from_scene(sc, solver_spec=spec).to_device()
        ens.tuning = {int(k): TuneConfig(cfg.threads, min(cfg.slots, 32 // int(k)) if cfg.slots else 0,
                                         cfg.min_blocks) for k in np.unique(sc.K)}
        ens.solve(200_000)
        torch.cuda.synchronize()
        _compare(href, ens.to_host())


@pytest.mark.gpu
def test_tuner_picks_and_solves_identically(cuda, tmp_path):
    import torch
    sc = scenes.mixed_k(ns=3000, span=(2.0, 4.0), seed=62)
    ens = Ensemble.from_scene(sc).to_device()
    tuner = autotune.Autotuner(slice_s=0.005, cache=str(tmp_path / "c.json"))
    table = tuner.tune(ens)
    assert set(table) == set(int(k) for k in np.unique(sc.K))
    assert ens.tuning == table
    assert all(v["rates"] for v in tuner.report.values())
    again = autotune.Autotuner(slice_s=0.005, cache=str(tmp_path / "c.json"))
    assert again.tune(Ensemble.from_scene(sc).to_device()) == table          # from the cache
    assert all(v["cached"] for v in again.report.values())
    ens.solve(300)
    ref = Ensemble.from_scene(sc).to_device()
    ref.solve(300)
    torch.cuda.synchronize()
    _compare(ref.to_host(), ens.to_host())
