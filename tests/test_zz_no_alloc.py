"""cbc_ensemble_solve_noalloc is for callers that cannot allocate device
memory while they step (their GPU memory belongs to another allocator or a
fixed budget); its scheduling scratch is a static device array of the
library, so nothing is allocated per call.  It gives bit-identical results to
cbc_ensemble_solve, over two calls in a row (the second resumes where the
first stopped), with and without a time slice.  Kept in its own file, named to
be collected last, so that it also runs after every other test in one process
(the scratch address is looked up once per device, by cbc_create, and then
reused).  A further test checks the claim itself: over warm calls, free
device memory and the torch allocator's counters do not move."""
import ctypes

import numpy as np
import pytest

from cbc_b200 import _lib, scenes
from cbc_b200.ensemble import Ensemble, make_work_list

pytestmark = pytest.mark.gpu

KEYS = ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters")


def _solve(ens, entry, max_steps, budget_ns=0, steps_total=False):
    import torch
    ctx = _lib.default_context(ens.device)
    spec, e = ens.spec(), ens.abi()
    w, keep = ens.work(make_work_list(ens.host["K"], ens.host["t_end"] - ens.host["t"]), budget_ns, steps_total)
    st = torch.cuda.current_stream(ens.device)
    fn = getattr(_lib.lib(), entry)
    ctx.check(fn(ctx.handle, ctypes.byref(spec), ctypes.byref(e), ctypes.byref(w), int(max_steps),
                 ctypes.c_void_p(st.cuda_stream)))
    torch.cuda.synchronize(ens.device)
    del keep


def _compare(ha, hb):
    for k in KEYS:
        x, y = ha[k], hb[k]
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert np.all(same), f"{k}: {np.count_nonzero(~same)} mismatches"


def test_noalloc_matches_ensemble_solve_two_calls(cuda):
    """Two calls in a row of 80 steps each; compared after each call."""
    sc = scenes.mixed_k(ns=400, span=(0.3, 1.2), seed=31)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    for _ in range(2):
        _solve(a, "cbc_ensemble_solve", 80)
        _solve(b, "cbc_ensemble_solve_noalloc", 80)
        _compare(a.to_host(), b.to_host())
    assert np.any(b.to_host()["steps"] > 80)


def _until_done(ens, entry, cap, budget_ns):
    calls = 0
    while calls < 2000:
        _solve(ens, entry, cap, budget_ns, steps_total=True)
        calls += 1
        st, steps = ens.dev["status"].cpu().numpy(), ens.dev["steps"].cpu().numpy()
        if not np.any(((st == 0) | (st == -1)) & (steps < cap)):
            break
    return calls


def test_noalloc_time_slices_match_ensemble_solve(cuda):
    """Device-time slices (the epoch word of the scratch) with a total step
    cap: where a deadline stops each system differs from run to run, the
    completed result does not."""
    sc = scenes.mixed_k(ns=400, span=(0.3, 1.2), seed=33)
    a = Ensemble.from_scene(sc).to_device()
    b = Ensemble.from_scene(sc).to_device()
    _until_done(a, "cbc_ensemble_solve", 300, 200_000)
    calls = _until_done(b, "cbc_ensemble_solve_noalloc", 300, 200_000)
    assert calls >= 2
    _compare(a.to_host(), b.to_host())


def test_noalloc_rejects_too_many_buckets(cuda):
    sc = scenes.mixed_k(ns=16, span=(0.3, 0.3), seed=32)
    ens = Ensemble.from_scene(sc).to_device()
    ctx = _lib.default_context(ens.device)
    spec, e = ens.spec(), ens.abi()
    w, keep = ens.work()
    w.nbuckets = 33                      # beyond the 32 cursors of the static scratch
    rc = _lib.lib().cbc_ensemble_solve_noalloc(ctx.handle, ctypes.byref(spec), ctypes.byref(e), ctypes.byref(w),
                                               10, None)
    assert rc == -1
    assert b"bucket" in _lib.lib().cbc_last_error(ctx.handle)
    del keep


def test_noalloc_warm_calls_allocate_nothing(cuda):
    """After one warm-up call (which may load the bucket kernels lazily), ten
    more calls leave the device's free memory and torch's allocator counters
    exactly where they were.  The ABI structures and the work list are built
    once, outside the measured region, as an allocation-free caller would."""
    import torch
    sc = scenes.mixed_k(ns=200, span=(0.2, 0.4), seed=34)
    ens = Ensemble.from_scene(sc).to_device()
    ctx = _lib.default_context(ens.device)
    spec, e = ens.spec(), ens.abi()
    w, keep = ens.work(make_work_list(ens.host["K"], ens.host["t_end"] - ens.host["t"]))
    st = torch.cuda.current_stream(ens.device)
    fn = _lib.lib().cbc_ensemble_solve_noalloc

    def call():
        ctx.check(fn(ctx.handle, ctypes.byref(spec), ctypes.byref(e), ctypes.byref(w), 40,
                     ctypes.c_void_p(st.cuda_stream)))

    call()
    torch.cuda.synchronize(ens.device)
    free0, _ = torch.cuda.mem_get_info(ens.device)
    stats0 = torch.cuda.memory_stats(ens.device)
    for _ in range(10):
        call()
    torch.cuda.synchronize(ens.device)
    free1, _ = torch.cuda.mem_get_info(ens.device)
    stats1 = torch.cuda.memory_stats(ens.device)
    assert free1 == free0
    for k in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current"):
        assert stats1.get(k, 0) == stats0.get(k, 0), k
    assert np.all(ens.dev["steps"].cpu().numpy() > 0)
    del keep
