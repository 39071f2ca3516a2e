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


def cost_weight(K: np.ndarray) -> np.ndarray:
    """Relative work of one step of a K-bubble system: RHS per bubble plus
    K^2 coupling pairs, each over ~14 Richardson sweeps."""
    K = np.asarray(K, dtype=np.float64)
    return 130.0 * K + 35.0 * K ** 2 + 14.0 * (20.0 * K ** 2 + 12.0 * K)


def make_work_list(K: np.ndarray, span: np.ndarray, active: Optional[np.ndarray] = None) -> WorkList:
    """Buckets of equal K, most expensive bucket first; inside a bucket the
    systems with the longest remaining span come first (longest-processing-
    time-first keeps the final tail short)."""
    K = np.asarray(K)
    idx_all = np.arange(K.shape[0]) if active is None else np.nonzero(active)[0]
    ks = np.unique(K[idx_all])
    ks = ks[np.argsort(-cost_weight(ks), kind="stable")]
    order: List[np.ndarray] = []
    begins = [0]
    for k in ks:
        sel = idx_all[K[idx_all] == k]
        sel = sel[np.argsort(-span[sel], kind="stable")]
        order.append(sel)
        begins.append(begins[-1] + sel.size)
    return WorkList(order=np.concatenate(order).astype(np.int32) if order else np.zeros(0, np.int32),
                    bucket_K=ks.astype(np.int32), bucket_begin=np.asarray(begins, dtype=np.int32))


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

    def scheduled_plan(self, max_steps: int = 1_000_000, pilot_steps: int = 256) -> "ScheduledPlan":
        if not self.dev:
            self.to_device()
        return ScheduledPlan(self, max_steps, pilot_steps)


class ScheduledPlan:
    """Two-phase batched solve with measured longest-first ordering.

    Phase 1 (pilot) advances every system by at most ``pilot_steps`` steps.
    The step rate it measures predicts each system's remaining work,
    (t_end - t) * pilot_steps / (t - t_start).  On the device, each K bucket
    of the phase-2 work list is re-sorted by that prediction (longest first,
    finished systems last), and phase 2 spends the rest of the budget.  Every
    call resumes exactly where the previous one stopped, so the results are
    bit-identical to a single solve with the same total budget; only the
    order in which warps pick up systems changes, which shortens the tail.
    ``launch()`` = pilot graph + a few sort kernels + main graph, all on one
    stream without host synchronisation.
    """

    def __init__(self, ens: Ensemble, max_steps: int, pilot_steps: int = 256):
        import torch
        if pilot_steps >= max_steps:
            raise ValueError("pilot_steps must be smaller than max_steps")
        self.ens = ens
        self.pilot_steps = int(pilot_steps)
        wl = make_work_list(ens.host["K"], ens.host["t_end"] - ens.host["t"])
        self.pilot = Plan(ens, self.pilot_steps, wl)
        main_wl = WorkList(order=wl.order.copy(), bucket_K=wl.bucket_K, bucket_begin=wl.bucket_begin)
        self.main = Plan(ens, int(max_steps) - self.pilot_steps, main_wl)
        dev = torch.device("cuda", ens.device)
        self.order_dev = self.main._keep[0]          # the main plan's device order array
        K = ens.host["K"]
        rank = np.empty(ens.ns, dtype=np.int64)
        for b, k in enumerate(wl.bucket_K):
            rank[K == k] = b
        self.bucket_rank = torch.from_numpy(rank).to(dev)
        self.t_start = torch.empty(ens.ns, dtype=torch.float64, device=dev)

    def launch(self, stream=None) -> None:
        import torch
        d = self.ens.dev
        st = stream if stream is not None else torch.cuda.current_stream(self.ens.device)
        with torch.cuda.stream(st):
            self.t_start.copy_(d["t"])
            self.pilot.launch(st)
            adv = (d["t"] - self.t_start).clamp(min=1e-300)
            remaining = (d["t_end"] - d["t"]).clamp(min=0.0) * (self.pilot_steps / adv)
            remaining = torch.where(d["status"] == -1, remaining, torch.zeros_like(remaining))
            by_cost = torch.sort(-remaining, stable=True).indices
            by_bucket = torch.sort(self.bucket_rank[by_cost], stable=True).indices
            self.order_dev.copy_(by_cost[by_bucket].to(torch.int32))
            self.main.launch(st)

    def close(self) -> None:
        self.pilot.close()
        self.main.close()


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
