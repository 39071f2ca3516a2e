"""The two-phase scheduled batched solve (pilot pass, device-side
longest-first re-ordering, main pass) is bit-identical to a single solve."""
import numpy as np
import pytest

from cbc_b200 import scenes
from cbc_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def test_scheduled_equals_single(cuda):
    import torch
    sc = scenes.mixed_k(ns=400, span=(0.2, 1.0), seed=21)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    a.plan(200_000).launch()
    sp = b.scheduled_plan(200_000, pilot_steps=64)
    sp.launch()
    torch.cuda.synchronize()
    ha, hb = a.to_host(), b.to_host()
    for k in ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
        x, y = ha[k], hb[k]
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert np.all(same), k
    sp.close()
