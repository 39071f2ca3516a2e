"""Continuous-batching solve server on one GPU.

Requests (one CKM1D system each: K bubbles, radii, drive, positions, span)
arrive at any time.  The server keeps a device-resident slot pool per K
bucket (a ragged ensemble preallocated once) and runs a loop of

  1. admit  -- queued requests whose bucket has a free slot are written into
               free slots (parameter precompute on the host, one batched
               host->device copy per bucket),
  2. advance -- one batched solve over all occupied slots with a bounded step
               budget per system (``chunk_steps``); systems resume exactly where
               the previous chunk stopped, so a request's result does not depend
               on what else is in flight,
  3. harvest -- statuses of the occupied slots come back (a few bytes per
               slot); finished requests release their slot.

Requests that arrive while others are on the GPU are admitted as soon as
slots free up and their work overlaps on the device with everything else in
flight.  Latency = completion time - arrival time.  There is no reference
counterpart (the reference only runs fixed batches through Model.solve); the
per-system integration is the same kernel and arithmetic as every other path.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import scenes
from .ensemble import Ensemble, WorkList
from .models import SolverSpec


@dataclass
class Request:
    rid: int
    K: int
    R0: np.ndarray           # (K,) um
    PA: np.ndarray           # (nk,) bar
    PS: np.ndarray           # (nk,) phase / pi
    X0: np.ndarray           # (K,) dimensionless positions
    span: float              # periods
    arrival: float = 0.0     # seconds (server clock)
    done: float = -1.0
    slot: int = -1
    result: Optional[Dict[str, np.ndarray]] = None


class SolveServer:
    """Slot pool: ``slots[K]`` systems of K bubbles for every K bucket."""

    def __init__(self, slots: Dict[int, int], nk: int = 2, ac: str = "SW_A", freqs_khz=(25.0, 50.0),
                 chunk_steps: int = 2048, max_steps: int = 1_000_000, solver_spec: Optional[SolverSpec] = None,
                 device: int = 0, keep_results: bool = False):
        import torch
        self.nk, self.ac, self.freqs = nk, ac, tuple(freqs_khz)
        self.chunk_steps = int(chunk_steps)
        self.max_steps = int(max_steps)
        self.keep_results = keep_results
        self.device = device
        self.tdev = torch.device("cuda", device)
        ks = sorted(slots)
        Ks = np.concatenate([np.full(slots[k], k, np.int32) for k in ks])
        ns = Ks.size
        # placeholder systems; every slot is (re)written at admission
        sc = scenes.Scene(K=Ks, R0=[np.full(k, 5.0) for k in Ks], PA=np.zeros((nk, ns)),
                          FR=np.tile(np.asarray(freqs_khz)[:, None], (1, ns)), PS=np.zeros((nk, ns)),
                          X0=[np.linspace(-0.2, 0.2, k) if k > 1 else np.zeros(1) for k in Ks],
                          t_end=np.zeros(ns), ac=ac)
        self.ens = Ensemble.from_scene(sc, solver_spec=solver_spec, device=device)
        self.ens.host["t_end"][:] = 0.0
        self.ens.host["status"][:] = 1
        self.ens.to_device()
        self.bucket_of = {k: np.nonzero(Ks == k)[0] for k in ks}
        self.free = {k: deque(self.bucket_of[k].tolist()) for k in ks}
        self.busy: Dict[int, Request] = {}
        self.queue: Dict[int, deque] = {k: deque() for k in ks}
        self.completed: List[Request] = []
        self.steps_done = 0
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ---- client side ----
    def submit(self, req: Request) -> None:
        if req.K not in self.queue:
            raise ValueError(f"no slot bucket for K={req.K}")
        self.queue[req.K].append(req)

    # ---- loop ----
    def _admit(self) -> int:
        import torch
        d, h = self.ens.dev, self.ens.host
        admitted = 0
        for k, q in self.queue.items():
            n = min(len(q), len(self.free[k]))
            if n == 0:
                continue
            reqs = [q.popleft() for _ in range(n)]
            slots = np.asarray([self.free[k].popleft() for _ in range(n)], dtype=np.int64)
            sc = scenes.Scene(K=np.full(n, k, np.int32), R0=[r.R0 for r in reqs],
                              PA=np.stack([r.PA for r in reqs], 1), FR=np.tile(np.asarray(self.freqs)[:, None], (1, n)),
                              PS=np.stack([r.PS for r in reqs], 1), X0=[r.X0 for r in reqs],
                              t_end=np.asarray([r.span for r in reqs]), ac=self.ac)
            part = Ensemble.from_scene(sc, solver_spec=self.ens.solver_spec)
            rows = (h["bubble_offset"][slots][:, None] + np.arange(k)[None, :]).reshape(-1)
            crow = (h["coupling_offset"][slots][:, None] + np.arange(3 * k * k)[None, :]).reshape(-1)
            sl = torch.from_numpy(slots).to(self.tdev)
            rw = torch.from_numpy(rows).to(self.tdev)
            cr = torch.from_numpy(crow).to(self.tdev)
            P = part.host
            for name, idx in (("state", rw), ("unit_params", rw)):
                d[name].index_copy_(0, idx, torch.from_numpy(P[name]).to(self.tdev))
            d["coupling"].index_copy_(0, cr, torch.from_numpy(P["coupling"]).to(self.tdev))
            for name in ("system_params", "control_params", "t", "t_end", "t_begin", "h", "event", "status",
                         "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
                d[name].index_copy_(0, sl, torch.from_numpy(P[name]).to(self.tdev))
            for r, s in zip(reqs, slots):
                r.slot = int(s)
                self.busy[int(s)] = r
            admitted += n
        return admitted

    def _advance(self) -> None:
        slots = np.fromiter(self.busy.keys(), dtype=np.int64)
        if slots.size == 0:
            return
        K = self.ens.host["K"][slots]
        ks = np.unique(K)
        order, begins = [], [0]
        for k in ks[::-1]:
            sel = slots[K == k]
            order.append(sel)
            begins.append(begins[-1] + sel.size)
        wl = WorkList(order=np.concatenate(order).astype(np.int32), bucket_K=ks[::-1].astype(np.int32),
                      bucket_begin=np.asarray(begins, np.int32))
        self.ens.solve(self.chunk_steps, work=wl)

    def _harvest(self) -> int:
        import torch
        slots = np.fromiter(self.busy.keys(), dtype=np.int64)
        if slots.size == 0:
            return 0
        idx = torch.from_numpy(slots).to(self.tdev)
        st = self.ens.dev["status"][idx].cpu().numpy()
        steps = self.ens.dev["steps"][idx].cpu().numpy()
        # -1: chunk budget spent, still running -- unless the request's total
        # step budget is used up, then it finishes as MAX_STEPS_REACHED
        finished = slots[(st != -1) | (steps >= self.max_steps)]
        tnow = self.now()
        for s in finished:
            r = self.busy.pop(int(s))
            r.done = tnow
            if self.keep_results:
                r.result = self.result_of(int(s))
            self.free[r.K].append(int(s))
            self.completed.append(r)
        return int(finished.size)

    def result_of(self, slot: int) -> Dict[str, np.ndarray]:
        h = self.ens.host
        k = int(h["K"][slot])
        b0 = int(h["bubble_offset"][slot])
        d = self.ens.dev
        return {"state": d["state"][b0:b0 + k].cpu().numpy(), "t": float(d["t"][slot]),
                "status": int(d["status"][slot]), "steps": int(d["steps"][slot]), "h": float(d["h"][slot])}

    def step(self) -> int:
        """One admit/advance/harvest iteration; returns completions."""
        self._admit()
        self._advance()
        return self._harvest()

    def idle(self) -> bool:
        return not self.busy and all(len(q) == 0 for q in self.queue.values())


def latency_stats(done: List[Request]) -> Dict[str, float]:
    lat = np.asarray([r.done - r.arrival for r in done])
    if lat.size == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p95_ms": float(np.percentile(lat, 95) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "completed": int(lat.size)}
