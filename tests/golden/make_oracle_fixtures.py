"""Generate the oracle fixtures of the full-size parity tests.

Test infrastructure.  Runs the CPU oracle (oracle/ckm1d_oracle.cpp, itself
pinned to the reference by the golden_ref_numba*.npz vectors) on two of the
headline workloads, at sizes that take the oracle minutes rather than the
seconds a GPU test may spend on it, and stores what the GPU tests compare
against in ``oracle_configs.npz``:

* ``large_k``: 256 systems of K = 32 bubbles (seed 4, R0 ~ U[2, 8] um,
  PA ~ U[0, 1.2] bar, positions inside one wavelength), 2 periods, 64
  samples per period (129 dense samples, reference schedule).  The dense
  output is 8.5 MB, so the fixture holds a SHA-256 digest of every output
  buffer (reference layout, NaNs canonicalised) plus the end state and the
  counters in full for diagnosis.
* ``mixed_k_2048``: 2,049 systems (2,048 split over K by its weights, each
  count rounded) drawn from the 65,536-system mixed-K ensemble (seed 1),
  stratified by K in proportion to its weights and, inside
  each K, evenly over the sorted spans, so spans run the whole 5-50 period
  range.  End state, times, step sizes, event values, statuses and counters
  are stored in full (ragged layout).

Both use max_steps = 1,000,000 (the headline benchmark's step cap).
Regenerate with ``python tests/golden/make_oracle_fixtures.py`` (about ten
minutes on 8 cores); the result does not depend on the machine (the oracle
is IEEE-deterministic: explicit fma, own elementary functions).
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (os.path.join(ROOT, "coupled-bubble-control_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

MAX_STEPS = 1_000_000
OUT = os.path.join(HERE, "oracle_configs.npz")

LARGE_K = dict(ns=256, K=32, periods=2.0, samples_per_period=64, seed=4)
MIXED_N = 2048
MIXED_SEED = 1

REF_KEYS = ("actual_time", "time_step", "actual_state", "actual_event", "status_flags", "dense_index",
            "dense_time", "dense_state", "total_steps", "rejected_steps", "convergece_success",
            "convergence_failures", "lin_iters")
RAGGED_KEYS = ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters")


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's bytes (C order), NaNs replaced by one canonical
    quiet NaN, prefixed by dtype and shape."""
    a = np.ascontiguousarray(a)
    if a.dtype.kind == "f":
        a = np.where(np.isnan(a), np.float64("nan"), a).astype(a.dtype)
    h = hashlib.sha256(a.tobytes()).hexdigest()
    return f"{a.dtype.str}{list(a.shape)}:{h}"


def large_k_scene():
    from cbc_b200 import scenes
    return scenes.large_k(ns=LARGE_K["ns"], K=LARGE_K["K"], periods=LARGE_K["periods"],
                          samples_per_period=LARGE_K["samples_per_period"], seed=LARGE_K["seed"])


def mixed_subset_indices(scene, n=MIXED_N):
    """Stratified by K (weights of the workload) and by span within each K."""
    from cbc_b200 import scenes
    idx = []
    for k, p in zip(scenes.MIXED_K, scenes.MIXED_P):
        sel = np.nonzero(scene.K == k)[0]
        sel = sel[np.argsort(scene.t_end[sel], kind="stable")]
        m = int(round(n * p))
        pick = np.unique(np.round(np.linspace(0, sel.size - 1, m)).astype(np.int64))
        idx.append(sel[pick])
    return np.sort(np.concatenate(idx))


def mixed_subset_scene():
    from cbc_b200 import scenes
    full = scenes.mixed_k(ns=65536, seed=MIXED_SEED)
    idx = mixed_subset_indices(full)
    return scenes.subset(full, idx), idx


def run_large_k(nthreads=0):
    from cbc_b200 import scenes
    from oracle import oracle
    m = scenes.build_model(large_k_scene())
    buf = oracle.solve_model(m, max_steps=MAX_STEPS, kernel_steps=MAX_STEPS, nthreads=nthreads)
    return buf


def run_mixed(nthreads=0):
    """Oracle end state of the mixed-K subset, scattered into the ragged layout."""
    from cbc_b200.ensemble import Ensemble
    from oracle import oracle
    import copy
    sc, idx = mixed_subset_scene()
    ens, models = Ensemble.from_scene(sc, return_models=True)
    out = {k: np.array(ens.host[k], copy=True) for k in RAGGED_KEYS}
    for k, (sel, m) in models.items():
        buf = copy.deepcopy(oracle.model_buffers(m))
        es, ms = m._execution_spec, m._model_spec
        spec = oracle.make_spec(es.ns, es.ups, es.tile, 0, ms.nk, ms.ac, ens.solver_spec)
        oracle.solve_ref_layout(spec, buf, MAX_STEPS, nthreads)
        bb = ens.host["bubble_offset"][sel][:, None] + np.arange(k)[None, :]
        out["state"][bb, :] = np.transpose(buf["actual_state"][:, :, :k], (1, 2, 0))
        out["t"][sel] = buf["actual_time"]
        out["h"][sel] = buf["time_step"]
        out["event"][sel] = buf["actual_event"]
        out["status"][sel] = buf["status_flags"]
        out["steps"][sel] = buf["total_steps"]
        out["rejected"][sel] = buf["rejected_steps"]
        out["conv_ok"][sel] = buf["convergece_success"]
        out["conv_fail"][sel] = buf["convergence_failures"]
        out["lin_iters"][sel] = buf["lin_iters"]
    return out, idx


def main():
    res = {}
    t0 = time.time()
    buf = run_large_k()
    for k in REF_KEYS:
        res[f"large_k/digest/{k}"] = np.array(digest(buf[k]))
    for k in ("actual_time", "time_step", "actual_state", "actual_event", "status_flags", "dense_index",
              "total_steps", "rejected_steps", "lin_iters"):
        res[f"large_k/end/{k}"] = buf[k]
    print(f"large_k: {time.time() - t0:.0f} s, steps {int(buf['total_steps'].sum())}", flush=True)
    t0 = time.time()
    out, idx = run_mixed()
    res["mixed_k_2048/index"] = idx
    for k, v in out.items():
        res[f"mixed_k_2048/end/{k}"] = v
    print(f"mixed_k_2048: {time.time() - t0:.0f} s, steps {int(out['steps'].sum())}, statuses "
          f"{dict(zip(*np.unique(out['status'], return_counts=True)))}", flush=True)
    np.savez_compressed(OUT, **res)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
