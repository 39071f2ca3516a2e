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


def test_latency_lanes_equal_single(cuda):
    """Systems moved into latency lanes (exclusive SMs) give the same results."""
    import torch
    from cbc_b200.ensemble import make_work_list, with_latency_lane
    sc = scenes.mixed_k(ns=300, span=(0.2, 0.8), seed=22)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    a.solve(200_000)
    span = b.host["t_end"] - b.host["t"]
    wl = with_latency_lane(make_work_list(b.host["K"], span), b.host["K"], span, fraction=0.1, max_sms=6)
    assert wl.exclusive is not None and 1 <= int(wl.exclusive.sum()) <= 6
    b.solve(200_000, work=wl)
    torch.cuda.synchronize()
    ha, hb = a.to_host(), b.to_host()
    for k in ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
        x, y = ha[k], hb[k]
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert np.all(same), k


def _compare(ha, hb, keys=("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail",
                           "lin_iters")):
    for k in keys:
        x, y = ha[k], hb[k]
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert np.all(same), f"{k}: {np.count_nonzero(~same)} mismatches"


def test_time_sliced_adaptive_equals_single(cuda):
    """Stopping every system at device-time deadlines and re-planning between
    slices (latency lanes included) reproduces a single solve bit for bit."""
    import torch
    sc = scenes.mixed_k(ns=600, span=(0.5, 2.0), seed=23)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    a.solve(200_000)
    plan = b.adaptive_plan(200_000, slices=(0.002, 0.004, 0.008, 0.016), max_lane_sms=4)
    plan.launch()
    torch.cuda.synchronize()
    _compare(a.to_host(), b.to_host())
    assert len(plan.history) >= 2          # the solve really was split


def test_steps_total_cap_equals_single_call(cuda):
    """max_steps over accumulated steps: slices that stop systems part-way
    still cap each system at exactly max_steps in total."""
    import torch
    from cbc_b200.ensemble import make_work_list
    sc = scenes.mixed_k(ns=200, span=(2.0, 4.0), seed=24)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    a.solve(150)
    wl = make_work_list(b.host["K"], b.host["t_end"] - b.host["t"])
    calls = 0
    while calls < 2000:
        b.solve(150, work=wl, budget_ns=300_000, steps_total=True)
        calls += 1
        st, steps = b.dev["status"].cpu().numpy(), b.dev["steps"].cpu().numpy()
        if not np.any(((st == 0) | (st == -1)) & (steps < 150)):
            break
    torch.cuda.synchronize()
    hb = b.to_host()
    assert calls > 1                       # the deadline did split the work
    assert np.all(hb["steps"] <= 150)
    _compare(a.to_host(), hb)


def test_plans_on_a_side_stream_equal_default_stream(cuda):
    """ScheduledPlan and AdaptivePlan given a non-default stream: the work-list
    upload, the state reads and the timing events follow that stream, so the
    results equal the default-stream solve bit for bit."""
    import torch
    sc = scenes.mixed_k(ns=300, span=(0.3, 1.0), seed=25)
    a = Ensemble.from_scene(sc).to_device()
    a.solve(200_000)
    torch.cuda.synchronize()
    ref = a.to_host()
    side = torch.cuda.Stream()
    b = Ensemble.from_scene(sc).to_device()
    torch.cuda.synchronize()
    sp = b.scheduled_plan(200_000, pilot_steps=48)
    sp.launch(stream=side)
    side.synchronize()
    _compare(ref, b.to_host())
    sp.close()
    c = Ensemble.from_scene(sc).to_device()
    torch.cuda.synchronize()
    ap = c.adaptive_plan(200_000, slices=(0.002, 0.004), max_lane_sms=2)
    ap.launch(stream=side)
    side.synchronize()
    _compare(ref, c.to_host())
    assert all(h.get("device_s", 0.0) >= 0.0 for h in ap.history)
