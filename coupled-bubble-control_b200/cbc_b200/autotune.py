"""Autotuner of the batched kernels' launch shape, per K bucket.

The reference fixes its launch shape at kernel-build time from the model's
specs: TILE = next_pow2(K) threads per system and SPB systems per block
become compile-time macros, and the register cap is a build option
(``backends/cupy_cuda/kernel_loader.py:35-63``, ``models/specs.py:40-52``,
``max_registers`` in ``backends/cuda_opts.py:6-73``).  Here the kernels are
prebuilt for sm_100a and the shape is chosen at run time by measurement:

* ``threads``     threads per block (32 .. 128; K = 32 is cut further to the
                  warps whose shared memory fits);
* ``slots``       systems a warp holds (32 // K, or half of it: idle lanes
                  for less intra-warp divergence of the Richardson iteration);
* ``min_blocks``  the register-budget variant of the kernel (0: the
                  compiler's full budget; 1: one more resident block per SM,
                  fewer registers per thread), K <= 8.

For every K of a workload the tuner runs each candidate on that K's systems
for a short device-time slice (the solve stops every system after its
current step when the slice ends, cbc_work.budget_ns), from the same
initial state, and keeps the candidate with the most step attempts per
second.  Results never depend on the shape (per-system arithmetic is the
same in every lane arrangement), so tuning is free to change between runs.
The table is cached per device name, library version, harmonics count and
linear solver in a JSON file (``$CBC_TUNE_CACHE`` or
``~/.cache/cbc_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
from dataclasses import asdict, dataclass
from typing import Callable, Dict, Iterable, List, Optional

import numpy as np


@dataclass(frozen=True)
class TuneConfig:
    threads: int = 128
    slots: int = 0          # 0: 32 // K (every lane busy)
    min_blocks: int = 0

    def label(self) -> str:
        return f"t{self.threads}/s{self.slots}/r{self.min_blocks}"


DEFAULT = TuneConfig()


def candidates(K: int) -> List[TuneConfig]:
    """The search space for K bubbles per system; the default first."""
    K = int(K)
    full = 32 // K
    slot_opts = [0] + ([full // 2] if full >= 2 else [])
    mb_opts = (0, 1) if K <= 8 else (0,)
    thread_opts = (128, 64, 32) if K <= 16 else (128, 64)
    out = []
    for th in thread_opts:
        for sl in slot_opts:
            for mb in mb_opts:
                out.append(TuneConfig(th, sl, mb))
    return out


def choose(rates: Dict[TuneConfig, float], margin: float = 0.02) -> TuneConfig:
    """Best measured candidate; the default wins unless another beats it by
    more than `margin` (relative), so measurement noise does not flip it."""
    if not rates:
        return DEFAULT
    best = max(rates, key=lambda c: rates[c])
    base = rates.get(DEFAULT)
    if base is not None and rates[best] <= base * (1.0 + margin):
        return DEFAULT
    return best


def cache_path() -> str:
    p = os.environ.get("CBC_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "cbc_b200", "autotune.json")


def cache_key(device_name: str, version: int, nk: int, lin_solver: str, K: int) -> str:
    return f"{device_name}|v{version}|nk{nk}|{lin_solver}|K{int(K)}"


def load_cache(path: Optional[str] = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(table: Dict[str, dict], path: Optional[str] = None) -> None:
    path = path or cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"     # one per process: ranks of a job may save at once
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home only costs a re-tune next time


def tune_k(K: int, measure: Callable[[TuneConfig], float], repeats: int = 2) -> Dict:
    """Measures every candidate for K (best of `repeats`) and picks one."""
    rates: Dict[TuneConfig, float] = {}
    for cfg in candidates(K):
        rates[cfg] = max(measure(cfg) for _ in range(repeats))
    best = choose(rates)
    return {"config": best, "rates": {c.label(): r for c, r in rates.items()},
            "gain_vs_default": rates[best] / rates[DEFAULT] if rates.get(DEFAULT) else 1.0}


class Autotuner:
    """Chooses a TuneConfig per K for an ensemble's workload on one device."""

    def __init__(self, device: int = 0, slice_s: float = 0.03, cache: Optional[str] = None,
                 use_cache: bool = True):
        self.device = int(device)
        self.slice_s = float(slice_s)
        self.cache = cache
        self.use_cache = use_cache
        self.report: Dict[int, dict] = {}

    def _pilot(self, ens, K: int) -> Callable[[TuneConfig], float]:
        """Measure function for the systems of K in `ens`: step attempts per
        second of one time slice from the initial state."""
        import torch
        from .ensemble import WorkList

        ids = np.nonzero(ens.host["K"] == K)[0].astype(np.int32)
        span = ens.host["t_end"][ids] - ens.host["t"][ids]
        ids = ids[np.argsort(-span, kind="stable")]

        def measure(cfg: TuneConfig) -> float:
            wl = WorkList(order=ids, bucket_K=np.asarray([K], np.int32),
                          bucket_begin=np.asarray([0, ids.size], np.int32),
                          threads=np.asarray([cfg.threads], np.int32),
                          slots=np.asarray([cfg.slots if cfg.slots > 0 else 32 // K], np.int32),
                          min_blocks=np.asarray([cfg.min_blocks if K <= 8 else 0], np.int32))
            ens.reset_device()
            torch.cuda.synchronize(self.device)
            a0 = int((ens.dev["steps"][ids].long() + ens.dev["rejected"][ids].long()).sum().item())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ens.solve(10 ** 9, work=wl, budget_ns=int(self.slice_s * 1e9))
            e1.record()
            torch.cuda.synchronize(self.device)
            a1 = int((ens.dev["steps"][ids].long() + ens.dev["rejected"][ids].long()).sum().item())
            return (a1 - a0) / (e0.elapsed_time(e1) * 1e-3)

        return measure

    def tune(self, ens, Ks: Optional[Iterable[int]] = None, force: bool = False) -> Dict[int, TuneConfig]:
        """Tunes every K of `ens` (or `Ks`), sets ens.tuning and returns it.
        The ensemble's device state is reset to its initial host values."""
        import torch
        from . import _lib
        if not ens.dev:
            ens.to_device()
        name = torch.cuda.get_device_name(self.device)
        version = int(_lib.lib().cbc_version())
        lin = ens.solver_spec.lin_solver
        table = load_cache(self.cache) if self.use_cache else {}
        out: Dict[int, TuneConfig] = {}
        saved_tuning = dict(ens.tuning)
        ens.tuning = {}
        for K in sorted(int(k) for k in (Ks if Ks is not None else np.unique(ens.host["K"]))):
            key = cache_key(name, version, ens.nk, lin, K)
            hit = table.get(key)
            if hit is not None and not force:
                out[K] = TuneConfig(**hit["config"])
                self.report[K] = dict(hit, cached=True)
                continue
            res = tune_k(K, self._pilot(ens, K))
            out[K] = res["config"]
            entry = {"config": asdict(res["config"]), "rates": res["rates"],
                     "gain_vs_default": res["gain_vs_default"]}
            table[key] = entry
            self.report[K] = dict(entry, cached=False)
        ens.reset_device()
        if self.use_cache:
            save_cache(table, self.cache)
        ens.tuning = {**saved_tuning, **out}
        return out

    def summary(self) -> Dict[str, dict]:
        return {f"K{k}": {"config": TuneConfig(**v["config"]).label() if isinstance(v["config"], dict)
                          else v["config"].label(),
                          "gain_vs_default": round(float(v["gain_vs_default"]), 4), "cached": v["cached"]}
                for k, v in sorted(self.report.items())}
