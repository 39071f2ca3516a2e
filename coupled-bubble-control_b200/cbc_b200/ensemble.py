"""Batched mixed-K ensembles resident on the GPU.

The reference integrates one ensemble shape (NS systems of exactly K
bubbles) per kernel build.  ``Ensemble`` holds systems of any K <= 32 in one
ragged set of device arrays (layout in include/cbc_b200.h, ``cbc_ensemble``)
and solves them all with one persistent work-stealing kernel per K bucket,
captured in a CUDA graph (``Ensemble.plan``).

Parameters are produced by the same precompute as the reference model
(``CKM1D.build_parameters``, reference models/ckm1d.py:133-202), run once per
K bucket, then scattered into the ragged arrays, so the ensemble and the
reference-layout path see bit-identical inputs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import _lib, scenes
from .models import SolverSpec

UP_STRIDE = 16   # unit_params row (13 used): 128-byte rows
SP_STRIDE = 8    # system_params row (5 used)


@dataclass
class WorkList:
    order: np.ndarray          # (n,) int32 system ids grouped by bucket
    bucket_K: np.ndarray       # (nb,) int32
    bucket_begin: np.ndarray   # (nb + 1,) int32
    threads: Optional[np.ndarray] = None
    blocks_per_sm: Optional[np.ndarray] = None
    share: Optional[np.ndarray] = None   # (nb,) float32 fraction of the GPU per bucket at the start


# Steady-state cost of one system-step on a full B200 (ns), measured on
# ensembles of identical systems (no tail); other K are interpolated.
STEP_NS = {1: 0.6, 2: 0.995, 3: 2.65, 4: 3.13, 6: 9.24, 8: 12.6}


def cost_weight(K) -> np.ndarray:
    """Relative cost of one step of a K-bubble system (ns on a full GPU)."""
    K = np.atleast_1d(np.asarray(K, dtype=np.float64))
    ks = np.asarray(sorted(STEP_NS), dtype=np.float64)
    vs = np.asarray([STEP_NS[int(k)] for k in ks])
    out = np.interp(K, ks, vs)
    big = K > ks[-1]
    out[big] = vs[-1] * (K[big] / ks[-1]) ** 2
    return out


def make_work_list(K: np.ndarray, work: np.ndarray, active: Optional[np.ndarray] = None,
                   shares: bool = True) -> WorkList:
    """Buckets of equal K, most expensive bucket first; inside a bucket the
    systems with the most predicted work come first (longest-processing-time
    first keeps the final tail short).  ``work`` is any per-system estimate of
    remaining steps (span, or span x measured step rate).  With ``shares``,
    every bucket starts at once with a fraction of the GPU proportional to its
    predicted cost (sum of work x cost per step)."""
    K = np.asarray(K)
    work = np.asarray(work, dtype=np.float64)
    idx_all = np.arange(K.shape[0]) if active is None else np.nonzero(active)[0]
    ks = np.unique(K[idx_all])
    ks = ks[np.argsort(-cost_weight(ks), kind="stable")]
    order: List[np.ndarray] = []
    begins = [0]
    cost = []
    for k in ks:
        sel = idx_all[K[idx_all] == k]
        sel = sel[np.argsort(-work[sel], kind="stable")]
        order.append(sel)
        begins.append(begins[-1] + sel.size)
        cost.append(float(np.sum(work[sel])) * float(cost_weight(k)[0]))
    sh = None
    if shares and len(ks) > 1:
        c = np.asarray(cost)
        sh = (c / c.sum()).astype(np.float32) if c.sum() > 0 else None
    return WorkList(order=np.concatenate(order).astype(np.int32) if order else np.zeros(0, np.int32),
                    bucket_K=ks.astype(np.int32), bucket_begin=np.asarray(begins, dtype=np.int32), share=sh)


class Ensemble:
    """Ragged ensemble: host numpy arrays plus torch device copies."""

    FIELDS_F64 = ("state", "unit_params", "system_params", "control_params", "coupling", "t", "t_end",
                  "t_begin", "h", "event")
    FIELDS_I32 = ("status", "dense_index", "steps", "rejected", "conv_ok", "conv_fail")

    def __init__(self, host: Dict[str, np.ndarray], nk: int, ac: str, ndo: int,
                 solver_spec: Optional[SolverSpec] = None, device: int = 0):
        self.host = host
        self.nk, self.ac, self.ndo = int(nk), ac, int(ndo)
        self.solver_spec = solver_spec if solver_spec is not None else SolverSpec()
        self.device = device
        self.ns = int(host["K"].shape[0])
        self.nb = int(host["state"].shape[0])
        self.dev: Dict[str, object] = {}
        self._plans: List[object] = []

    # ---- construction ----
    @classmethod
    def from_scene(cls, scene: scenes.Scene, solver_spec: Optional[SolverSpec] = None,
                   ndo: Optional[int] = None, device: int = 0, return_models: bool = False):
        ndo = scene.ndo if ndo is None else int(ndo)
        K = scene.K.astype(np.int32)
        ns = K.shape[0]
        nk = scene.nk
        boff = np.zeros(ns, dtype=np.int64)
        boff[1:] = np.cumsum(K[:-1].astype(np.int64))
        nb = int(K.sum())
        coff = np.zeros(ns, dtype=np.int64)
        coff[1:] = np.cumsum(3 * K[:-1].astype(np.int64) ** 2)
        h = {
            "K": K, "bubble_offset": boff, "coupling_offset": coff,
            "state": np.zeros((nb, 4)), "unit_params": np.zeros((nb, UP_STRIDE)),
            "system_params": np.zeros((ns, SP_STRIDE)), "control_params": np.zeros((ns, 4 * nk)),
            "coupling": np.zeros(int(np.sum(3 * K.astype(np.int64) ** 2))),
            "t": np.zeros(ns), "t_end": np.zeros(ns), "t_begin": np.zeros(ns), "h": np.zeros(ns),
            "event": np.zeros(ns), "status": np.zeros(ns, np.int32), "dense_index": np.zeros(ns, np.int32),
            "steps": np.zeros(ns, np.int32), "rejected": np.zeros(ns, np.int32),
            "conv_ok": np.zeros(ns, np.int32), "conv_fail": np.zeros(ns, np.int32),
            "lin_iters": np.zeros(ns, np.int64),
            "dense_time": np.zeros((max(ndo, 0), ns)), "dense_state": np.zeros((max(ndo, 0), nb, 4)),
        }
        models = {}
        for k in np.unique(K):
            sel = np.nonzero(K == k)[0]
            sub = scenes.subset(scene, sel)
            m = scenes.build_model(sub, solver_spec=solver_spec, ndo=0)
            models[int(k)] = (sel, m)
            hb = m.runtime.host_buffers
            st, pr, su = hb.state, hb.params, hb.status
            bb = boff[sel][:, None] + np.arange(k)[None, :]                    # (n, k) bubble rows
            h["state"][bb, :] = np.transpose(st.actual_state[:, :, :k], (1, 2, 0))
            h["unit_params"][bb, :13] = np.transpose(pr.unit_params[:, :, :k], (1, 2, 0))
            h["system_params"][sel, :5] = pr.system_params.T
            h["control_params"][sel, :] = pr.control_params.T
            blk = np.transpose(pr.coupling_matrices[:, :, :, :k], (2, 0, 1, 3)).reshape(sel.size, -1)
            cidx = coff[sel][:, None] + np.arange(3 * k * k)[None, :]
            h["coupling"][cidx] = blk
            h["t"][sel] = st.actual_time
            h["t_end"][sel] = st.time_end
            h["t_begin"][sel] = st.time_begin
            h["h"][sel] = st.time_step
            h["event"][sel] = su.actual_event
        ens = cls(h, nk, scene.ac, ndo, solver_spec, device)
        return (ens, models) if return_models else ens

    # ---- device residency ----
    def to_device(self) -> "Ensemble":
        import torch
        dev = torch.device("cuda", self.device)
        self.dev = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in self.host.items()}
        return self

    def enable_trace(self) -> None:
        """Record per-system load / write-back GPU timestamps (ns) in
        dev['trace_load_ns'] / dev['trace_done_ns'] on later solves and plans."""
        import torch
        dev = torch.device("cuda", self.device)
        self.dev["trace_load_ns"] = torch.zeros(self.ns, dtype=torch.int64, device=dev)
        self.dev["trace_done_ns"] = torch.zeros(self.ns, dtype=torch.int64, device=dev)

    def reset_device(self) -> None:
        """Copy the host arrays (initial conditions) into the existing device arrays."""
        import torch
        for k, v in self.host.items():
            self.dev[k].copy_(torch.from_numpy(np.ascontiguousarray(v)))

    def to_host(self) -> Dict[str, np.ndarray]:
        return {k: v.cpu().numpy() for k, v in self.dev.items()}

    # ---- ABI structures ----
    def spec(self) -> _lib.cbc_spec:
        s = self.solver_spec
        return _lib.cbc_spec(self.ns, 0, 0, self.ndo, self.nk, _lib.AC_CODES[self.ac],
                             _lib.DENSE_CODES[s.dense_mode], int(s.lin_max_iter), s.atol, s.rtol, s.min_step,
                             s.max_step, s.lin_atol, s.lin_rtol, s.lin_relaxation, s.etol, s.col_threshold)

    def abi(self) -> _lib.cbc_ensemble:
        d = self.dev
        e = _lib.cbc_ensemble()
        e.ns, e.nb = self.ns, self.nb
        e.up_stride, e.sp_stride, e.cp_stride = UP_STRIDE, SP_STRIDE, 4 * self.nk
        for name in ("bubble_offset", "coupling_offset", "state", "unit_params", "system_params",
                     "control_params", "coupling", "t", "t_end", "t_begin", "h", "event", "status",
                     "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
            setattr(e, name, d[name].data_ptr())
        if "trace_load_ns" in d:
            e.trace_load_ns = d["trace_load_ns"].data_ptr()
            e.trace_done_ns = d["trace_done_ns"].data_ptr()
        if self.ndo > 0:
            e.dense_index = d["dense_index"].data_ptr()
            e.dense_time = d["dense_time"].data_ptr()
            e.dense_state = d["dense_state"].data_ptr()
        return e

    def work(self, wl: Optional[WorkList] = None):
        """(cbc_work, keep-alive list) for a work list (default: all systems)."""
        import torch
        if wl is None:
            wl = make_work_list(self.host["K"], self.host["t_end"] - self.host["t"])
        order = torch.from_numpy(wl.order).to(torch.device("cuda", self.device))
        keep = [order, wl]
        w = _lib.cbc_work()
        w.order = order.data_ptr()
        w.nbuckets = int(wl.bucket_K.size)
        bk = np.ascontiguousarray(wl.bucket_K, dtype=np.int32)
        bb = np.ascontiguousarray(wl.bucket_begin, dtype=np.int32)
        keep += [bk, bb]
        w.bucket_K = bk.ctypes.data
        w.bucket_begin = bb.ctypes.data
        if wl.threads is not None:
            th = np.ascontiguousarray(wl.threads, dtype=np.int32)
            keep.append(th)
            w.threads = th.ctypes.data
        if wl.blocks_per_sm is not None:
            bp = np.ascontiguousarray(wl.blocks_per_sm, dtype=np.int32)
            keep.append(bp)
            w.blocks_per_sm = bp.ctypes.data
        if wl.share is not None:
            sh = np.ascontiguousarray(wl.share, dtype=np.float32)
            keep.append(sh)
            w.share = sh.ctypes.data
        return w, keep

    # ---- solving ----
    def solve(self, max_steps: int = 1_000_000, work: Optional[WorkList] = None, stream=None) -> None:
        """Enqueue one batched solve on `stream` (default: current torch stream)."""
        import torch
        if not self.dev:
            self.to_device()
        ctx = _lib.default_context(self.device)
        spec, e = self.spec(), self.abi()
        w, keep = self.work(work)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        ctx.check(_lib.lib().cbc_ensemble_solve(ctx.handle, ctypes.byref(spec), ctypes.byref(e),
                                                ctypes.byref(w), int(max_steps), ctypes.c_void_p(st.cuda_stream)))
        self._keep = keep

    def plan(self, max_steps: int = 1_000_000, work: Optional[WorkList] = None) -> "Plan":
        if not self.dev:
            self.to_device()
        return Plan(self, max_steps, work)

    def scheduled_plan(self, max_steps: int = 1_000_000, pilot_steps: int = 2048) -> "ScheduledPlan":
        if not self.dev:
            self.to_device()
        return ScheduledPlan(self, max_steps, pilot_steps)


class ScheduledPlan:
    """Two-phase batched solve with measured longest-first ordering.

    Phase 1 (pilot, one graph launch) advances every system by at most
    ``pilot_steps`` steps.  The step rate it measures predicts each system's
    remaining steps, (t_end - t) * pilot_steps / (t - t_start).  Phase 2 solves
    the systems still running with every K bucket started at once, a GPU share
    per bucket proportional to its predicted cost, and each bucket's systems
    in longest-predicted-first order.  Every call resumes exactly where the
    previous one stopped, so the results are bit-identical to a single solve
    with the same total budget; only the order in which warps pick systems up
    changes, which shortens the tail.
    """

    def __init__(self, ens: Ensemble, max_steps: int, pilot_steps: int = 2048):
        if pilot_steps >= max_steps:
            raise ValueError("pilot_steps must be smaller than max_steps")
        self.ens = ens
        self.max_steps = int(max_steps)
        self.pilot_steps = int(pilot_steps)
        span = ens.host["t_end"] - ens.host["t"]
        self.pilot = Plan(ens, self.pilot_steps, make_work_list(ens.host["K"], span))
        self.last_work: Optional[WorkList] = None
        self.rate_clip = (200.0, 20000.0)   # steps per period

    def launch(self, stream=None) -> None:
        import torch
        d = self.ens.dev
        t_start = d["t"].clone()
        self.pilot.launch(stream)
        torch.cuda.synchronize(self.ens.device)
        t = d["t"].cpu().numpy()
        t0 = t_start.cpu().numpy()
        status = d["status"].cpu().numpy()
        t_end = d["t_end"].cpu().numpy()
        adv = np.maximum(t - t0, 1e-300)
        # a system caught in a collapse during the pilot advances very little:
        # clip its measured rate to a plausible range before extrapolating
        rate = np.clip(self.pilot_steps / adv, self.rate_clip[0], self.rate_clip[1])
        remaining = np.maximum(t_end - t, 0.0)
        pred = remaining * rate
        active = status == -1
        if not np.any(active):
            return
        K = self.ens.host["K"]
        wl = make_work_list(K, pred, active=active)
        # bucket shares from the remaining spans (robust); the measured rates
        # only order the systems inside each bucket
        span_wl = make_work_list(K, remaining, active=active)
        wl.share = span_wl.share
        self.last_work = wl
        self.ens.solve(self.max_steps - self.pilot_steps, work=wl, stream=stream)

    def close(self) -> None:
        self.pilot.close()


class Plan:
    """A captured CUDA graph of one batched solve bound to an ensemble's
    device arrays.  ``launch()`` replays it (a single graph launch)."""

    def __init__(self, ens: Ensemble, max_steps: int, work: Optional[WorkList]):
        self.ens = ens
        self.ctx = _lib.default_context(ens.device)
        self._spec, self._e = ens.spec(), ens.abi()
        self._w, self._keep = ens.work(work)
        h = _lib.P()
        self.ctx.check(_lib.lib().cbc_plan_create(self.ctx.handle, ctypes.byref(self._spec), ctypes.byref(self._e),
                                                  ctypes.byref(self._w), int(max_steps), ctypes.byref(h)))
        self.handle = h.value

    def launch(self, stream=None) -> None:
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.ens.device)
        self.ctx.check(_lib.lib().cbc_plan_launch(self.handle, ctypes.c_void_p(st.cuda_stream)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.lib().cbc_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
