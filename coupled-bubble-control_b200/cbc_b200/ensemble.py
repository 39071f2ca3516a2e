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
    exclusive: Optional[np.ndarray] = None   # (nb,) int32 SMs of a latency lane (0: ordinary bucket)
    slots: Optional[np.ndarray] = None       # (nb,) int32 systems per warp (autotuner)
    min_blocks: Optional[np.ndarray] = None  # (nb,) int32 register-budget variant 0 / 1 (autotuner)


# Steady-state cost of one step attempt on a full B200 (ns), measured on the
# K buckets of the mixed-K workload filling the GPU (a 0.5 s slice from t = 0;
# `python bench.py --workload costs`); other K are interpolated.
STEP_NS = {1: 0.58, 2: 0.846, 3: 2.14, 4: 2.55, 6: 6.32, 8: 7.16}
# Latency of one step attempt of a system whose warp has an SM sub-partition
# to itself (us), measured on single systems of the mixed-K workload.
ALONE_US = {1: 9.3, 2: 13.9, 3: 15.8, 4: 14.8, 6: 23.5, 8: 23.9}


def cost_weight(K) -> np.ndarray:
    """Relative cost of one step of a K-bubble system (ns on a full GPU)."""
    K = np.atleast_1d(np.asarray(K, dtype=np.float64))
    ks = np.asarray(sorted(STEP_NS), dtype=np.float64)
    vs = np.asarray([STEP_NS[int(k)] for k in ks])
    out = np.interp(K, ks, vs)
    big = K > ks[-1]
    out[big] = vs[-1] * (K[big] / ks[-1]) ** 2
    return out


def alone_latency(K) -> np.ndarray:
    """Per-attempt latency (us) of a K-bubble system running alone on an SM
    sub-partition; K > 8 extrapolated linearly in K."""
    K = np.atleast_1d(np.asarray(K, dtype=np.float64))
    ks = np.asarray(sorted(ALONE_US), dtype=np.float64)
    vs = np.asarray([ALONE_US[int(k)] for k in ks])
    out = np.interp(K, ks, vs)
    big = K > ks[-1]
    out[big] = vs[-1] * K[big] / ks[-1]
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


def with_latency_lane(wl: WorkList, K: np.ndarray, work: np.ndarray, fraction: float = 1e-3,
                      max_sms: int = 12) -> WorkList:
    """Moves the systems with the longest predicted serial time into latency
    lanes: extra buckets of the same K whose blocks (4 warps) each hold an SM
    alone, so their steps run at the minimum latency instead of sharing issue
    slots with a full SM.  The serial time of a system is its predicted steps
    times the per-step latency of its warp on a full GPU, which grows with the
    cost of one system-step and the number of systems a warp carries.  At most
    ``fraction`` of the systems and ``max_sms`` SMs are used."""
    K = np.asarray(K)
    work = np.asarray(work, dtype=np.float64)
    if wl.order.size == 0 or max_sms < 1:
        return wl
    ids = wl.order
    chain = work[ids] * cost_weight(K[ids]) * (32 // K[ids])
    n_lat = int(np.ceil(fraction * ids.size))
    top = ids[np.argsort(-chain, kind="stable")[:n_lat]]
    # trim to the SM budget, keeping the longest chains
    picked, count, sms = [], {}, {}
    used = 0
    for s_ in top:
        k = int(K[s_])
        opens_block = count.get(k, 0) % (4 * (32 // k)) == 0   # a new 4-warp block, one more SM
        if opens_block and used + 1 > max_sms:
            continue
        if opens_block:
            sms[k] = sms.get(k, 0) + 1
            used += 1
        count[k] = count.get(k, 0) + 1
        picked.append(int(s_))
    if not picked:
        return wl
    order, bk, bb = [], [], [0]
    share = [] if wl.share is not None else None
    excl = []
    for b in range(wl.bucket_K.size):
        seg = wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]]
        seg = seg[~np.isin(seg, picked)]
        order.append(seg)
        bk.append(int(wl.bucket_K[b]))
        bb.append(bb[-1] + seg.size)
        excl.append(0)
        if share is not None:
            share.append(float(wl.share[b]))
    for k in sorted(sms, key=lambda k: -cost_weight(k)[0]):
        sel = np.asarray([p for p in picked if int(K[p]) == k], dtype=np.int32)
        sel = sel[np.argsort(-work[sel], kind="stable")]
        order.append(sel)
        bk.append(k)
        bb.append(bb[-1] + sel.size)
        excl.append(sms[k])
        if share is not None:
            share.append(0.0)
    return WorkList(order=np.concatenate(order).astype(np.int32), bucket_K=np.asarray(bk, np.int32),
                    bucket_begin=np.asarray(bb, np.int32), threads=None, blocks_per_sm=None,
                    share=None if share is None else np.asarray(share, np.float32),
                    exclusive=np.asarray(excl, np.int32))


class Ensemble:
    """Ragged ensemble: host numpy arrays plus torch device copies."""

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
        # per-K launch shape chosen by cbc_b200.autotune (K -> TuneConfig);
        # applied to every work list that does not set its own
        self.tuning: Dict[int, object] = {}

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
                             s.max_step, s.lin_atol, s.lin_rtol, s.lin_relaxation, s.etol, s.col_threshold,
                             _lib.LIN_CODES[s.lin_solver], 0)

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

    def work(self, wl: Optional[WorkList] = None, budget_ns: int = 0, steps_total: bool = False, stream=None):
        """(cbc_work, keep-alive list) for a work list (default: all systems).
        The device copy of the order is made on `stream` (default: the current
        torch stream), so kernels later enqueued on that stream see it, and is
        marked in use by that stream for torch's caching allocator."""
        import torch
        if wl is None:
            wl = make_work_list(self.host["K"], self.host["t_end"] - self.host["t"])
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(st):
            order = torch.from_numpy(wl.order).to(torch.device("cuda", self.device), non_blocking=False)
        order.record_stream(st)
        keep = [order, wl]
        w = _lib.cbc_work()
        w.order = order.data_ptr()
        w.nbuckets = int(wl.bucket_K.size)
        bk = np.ascontiguousarray(wl.bucket_K, dtype=np.int32)
        bb = np.ascontiguousarray(wl.bucket_begin, dtype=np.int32)
        keep += [bk, bb]
        w.bucket_K = bk.ctypes.data
        w.bucket_begin = bb.ctypes.data
        if wl.blocks_per_sm is not None:
            bp = np.ascontiguousarray(wl.blocks_per_sm, dtype=np.int32)
            keep.append(bp)
            w.blocks_per_sm = bp.ctypes.data
        if wl.share is not None:
            sh = np.ascontiguousarray(wl.share, dtype=np.float32)
            keep.append(sh)
            w.share = sh.ctypes.data
        if wl.exclusive is not None:
            ex = np.ascontiguousarray(wl.exclusive, dtype=np.int32)
            keep.append(ex)
            w.exclusive = ex.ctypes.data
        tuned = self._tuned_arrays(wl)
        for name in ("threads", "slots", "min_blocks"):
            arr = getattr(wl, name, None)
            if arr is None:
                arr = tuned.get(name)
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.int32)
                keep.append(a)
                setattr(w, name, a.ctypes.data)
        w.budget_ns = int(budget_ns)
        w.steps_total = 1 if steps_total else 0
        return w, keep

    def _tuned_arrays(self, wl: WorkList) -> Dict[str, np.ndarray]:
        """threads / slots / min_blocks per bucket from self.tuning (latency
        lanes keep the defaults: whole warps, the full register budget)."""
        if not self.tuning:
            return {}
        nb = int(wl.bucket_K.size)
        th = np.full(nb, 128, np.int32)
        sl = np.asarray([32 // int(k) for k in wl.bucket_K], np.int32)
        mb = np.zeros(nb, np.int32)
        for b, k in enumerate(wl.bucket_K):
            cfg = self.tuning.get(int(k))
            if cfg is None or (wl.exclusive is not None and wl.exclusive[b] > 0):
                continue
            th[b] = cfg.threads
            sl[b] = cfg.slots if cfg.slots > 0 else 32 // int(k)
            mb[b] = cfg.min_blocks if int(k) <= 8 else 0
        return {"threads": th, "slots": sl, "min_blocks": mb}

    # ---- solving ----
    def solve(self, max_steps: int = 1_000_000, work: Optional[WorkList] = None, stream=None,
              budget_ns: int = 0, steps_total: bool = False) -> None:
        """Enqueue one batched solve on `stream` (default: current torch stream).
        budget_ns > 0 stops every system that long after the solve starts
        (resumable, status -1); steps_total makes max_steps a cap on the steps
        accumulated over all calls."""
        import torch
        if not self.dev:
            self.to_device()
        ctx = _lib.default_context(self.device)
        spec, e = self.spec(), self.abi()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        w, keep = self.work(work, budget_ns, steps_total, stream=st)
        ctx.check(_lib.lib().cbc_ensemble_solve(ctx.handle, ctypes.byref(spec), ctypes.byref(e),
                                                ctypes.byref(w), int(max_steps), ctypes.c_void_p(st.cuda_stream)))
        self._keep = keep

    def plan(self, max_steps: int = 1_000_000, work: Optional[WorkList] = None) -> "Plan":
        if not self.dev:
            self.to_device()
        return Plan(self, max_steps, work)

    def adaptive_plan(self, max_steps: int = 1_000_000, slices=(1.0, 2.0, 4.0, 8.0),
                      max_lane_sms: int = 32, load_factor: float = 1.2, solo: int = 0) -> "AdaptivePlan":
        if not self.dev:
            self.to_device()
        return AdaptivePlan(self, max_steps, slices, max_lane_sms, load_factor, solo)

    def scheduled_plan(self, max_steps: int = 1_000_000, pilot_steps: int = 2048,
                       latency_lane: bool = True) -> "ScheduledPlan":
        if not self.dev:
            self.to_device()
        return ScheduledPlan(self, max_steps, pilot_steps, latency_lane)


class ScheduledPlan:
    """Two-phase batched solve with measured longest-first ordering.

    Phase 1 (pilot, one graph launch) advances every system by at most
    ``pilot_steps`` steps.  The step rate it measures predicts each system's
    remaining steps, (t_end - t) * pilot_steps / (t - t_start).  Phase 2 solves
    the systems still running with every K bucket started at once, a GPU share
    per bucket proportional to its predicted cost, and each bucket's systems
    in longest-predicted-first order; the systems with the longest predicted
    serial time run in latency lanes (``with_latency_lane``).  Every call resumes exactly where the
    previous one stopped, so the results are bit-identical to a single solve
    with the same total budget; only the order in which warps pick systems up
    changes, which shortens the tail.
    """

    def __init__(self, ens: Ensemble, max_steps: int, pilot_steps: int = 2048, latency_lane: bool = True):
        if pilot_steps >= max_steps:
            raise ValueError("pilot_steps must be smaller than max_steps")
        self.ens = ens
        self.max_steps = int(max_steps)
        self.pilot_steps = int(pilot_steps)
        span = ens.host["t_end"] - ens.host["t"]
        self.pilot = Plan(ens, self.pilot_steps, make_work_list(ens.host["K"], span))
        self.last_work: Optional[WorkList] = None
        self.rate_clip = (200.0, 20000.0)   # steps per period
        self.latency_lane = bool(latency_lane)

    def launch(self, stream=None) -> None:
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.ens.device)
        with torch.cuda.stream(st):   # every torch op of the plan is ordered with its kernels
            self._launch(st)

    def _launch(self, stream) -> None:
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
        if self.latency_lane:
            wl = with_latency_lane(wl, K, pred)
        self.last_work = wl
        self.ens.solve(self.max_steps - self.pilot_steps, work=wl, stream=stream)

    def close(self) -> None:
        self.pilot.close()


def lane_work_list(wl: WorkList, K: np.ndarray, lane_ids: np.ndarray, order_key: np.ndarray,
                   sms_by_k: Dict[int, int], solo_ids=()) -> WorkList:
    """Moves the systems lane_ids out of the buckets of wl into latency lanes:
    one extra bucket per K with sms_by_k[K] exclusive SMs, longest order_key
    first.  Systems in solo_ids (a subset of lane_ids) get solo lanes: a
    bucket of their K whose warps hold one system each (slots = 1), so their
    Richardson loop never waits for warp-mates; four per exclusive SM."""
    lane_ids = np.asarray(lane_ids)
    solo_ids = np.asarray(solo_ids, dtype=np.int64)
    moved = lane_ids                        # every system leaving the ordinary buckets
    if solo_ids.size:
        moved = np.union1d(lane_ids, solo_ids)
        lane_ids = lane_ids[~np.isin(lane_ids, solo_ids)]
    order, bk, bb = [], [], [0]
    share = [] if wl.share is not None else None
    excl = []
    for b in range(wl.bucket_K.size):
        seg = wl.order[wl.bucket_begin[b]:wl.bucket_begin[b + 1]]
        seg = seg[~np.isin(seg, moved)]
        order.append(seg)
        bk.append(int(wl.bucket_K[b]))
        bb.append(bb[-1] + seg.size)
        excl.append(0)
        if share is not None:
            share.append(float(wl.share[b]))
    for k in sorted(sms_by_k, key=lambda k: -cost_weight(k)[0]):
        sel = lane_ids[K[lane_ids] == k]
        if sel.size == 0 or sms_by_k[k] < 1:
            continue
        sel = sel[np.argsort(-order_key[sel], kind="stable")]
        order.append(sel)
        bk.append(int(k))
        bb.append(bb[-1] + sel.size)
        excl.append(int(sms_by_k[k]))
        if share is not None:
            share.append(0.0)
    slots = [32 // int(k) for k in bk]
    for k in sorted(set(int(x) for x in K[solo_ids])) if solo_ids.size else []:
        sel = solo_ids[K[solo_ids] == k]
        sel = sel[np.argsort(-order_key[sel], kind="stable")]
        order.append(sel.astype(np.int32))
        bk.append(int(k))
        bb.append(bb[-1] + sel.size)
        excl.append(int((sel.size + 3) // 4))
        slots.append(1)
        if share is not None:
            share.append(0.0)
    return WorkList(order=np.concatenate(order).astype(np.int32), bucket_K=np.asarray(bk, np.int32),
                    bucket_begin=np.asarray(bb, np.int32),
                    share=None if share is None else np.asarray(share, np.float32),
                    exclusive=np.asarray(excl, np.int32),
                    slots=np.asarray(slots, np.int32) if solo_ids.size else None)


def adaptive_work_list(K, t_end, t0, a0, t, attempts, active, sm_count: int, max_lane_sms: int = 32,
                       load_factor: float = 1.2, min_observed: int = 256, solo: int = 0):
    """One re-planning step of ``AdaptivePlan`` (host only): the work list
    for the systems still running, from the progress since the solve began
    (t0 / a0: simulated time and step attempts then; t / attempts: now).
    Returns (work list, summary dict)."""
    K = np.asarray(K)
    ids = np.nonzero(active)[0]
    adv = t - t0
    obs = attempts - a0
    own = (obs >= min_observed) & (adv > 0)
    rate = np.zeros(K.shape[0])
    rate[own] = obs[own] / adv[own]
    for k in np.unique(K[ids]):
        sel = (K == k) & own
        fill = float(np.median(rate[sel])) if np.any(sel) else 2000.0
        rate[(K == k) & ~own] = fill
    remaining = rate * np.maximum(t_end - t, 0.0)
    serial_s = remaining * alone_latency(K) * 1e-6
    bulk_s = float(np.sum(remaining[ids] * cost_weight(K[ids]))) * 1e-9
    wl = make_work_list(K, remaining, active=active)
    # latency lanes for the systems that would otherwise end last
    lane_sms = 0
    picked: List[int] = []
    sms: Dict[int, int] = {}
    count: Dict[int, int] = {}
    for s in ids[np.argsort(-serial_s[ids], kind="stable")]:
        rest = sm_count - lane_sms
        if serial_s[s] * load_factor < bulk_s * sm_count / max(rest, 1):
            break
        k = int(K[s])
        opens = count.get(k, 0) % (4 * (32 // k)) == 0
        if opens and lane_sms + 1 > max_lane_sms:
            break
        if opens:
            sms[k] = sms.get(k, 0) + 1
            lane_sms += 1
        count[k] = count.get(k, 0) + 1
        picked.append(int(s))
    solo_ids = np.asarray(picked[:solo], dtype=np.int64)    # the longest chains run alone in their warp
    if picked:
        wl = lane_work_list(wl, K, np.asarray(picked), serial_s, sms, solo_ids=solo_ids)
    info = {"active": int(ids.size), "bulk_s": bulk_s, "lane_systems": len(picked), "lane_sms": lane_sms,
            "solo_systems": int(solo_ids.size),
            "max_serial_s": float(serial_s[ids].max()) if ids.size else 0.0}
    return wl, info


class AdaptivePlan:
    """Time-sliced batched solve that re-plans between slices.

    Which systems run longest cannot be told from their first steps: in the
    mixed-K workload a third of the K = 8 systems fail early (step-size
    limit, non-convergence, non-finite state) after stepping just as fast as
    the systems that run to the end.  Long systems reveal themselves by
    surviving.  So the solve runs in slices of device time (``slices``
    seconds, then one unbounded slice); every slice stops all systems after
    their current step (resumable, bit-identical), and the host re-plans the
    rest from the progress seen so far:

    * remaining attempts of a system = its observed attempts per unit of
      simulated time x its remaining span (the median rate of its K while it
      has not run enough steps to measure its own);
    * a system whose remaining attempts at the latency it sees outside a lane
      (its alone latency ``ALONE_US`` x ``load_factor``; the latency of one
      attempt inside the full GPU is 1.31-1.48x the alone latency for
      K = 3..8 on a full B200, ``bench.py --workload costs``, but 1.2 gave
      the shortest mixed-K solves of 1.0-1.35: every lane takes a whole SM
      from the bulk)
      exceed the predicted bulk time would end last: it goes to a latency
      lane (an SM of its own, ``cbc_work.exclusive``), longest first, up to
      ``max_lane_sms`` SMs;
    * every other system goes to its K bucket, longest first, with bucket
      shares proportional to the predicted cost (``STEP_NS``).

    max_steps caps the steps each system accumulates over all slices
    (``steps_total``), so the results equal one solve with that cap.
    """

    MIN_OBSERVED = 256   # attempts before a system's own rate is trusted

    def __init__(self, ens: Ensemble, max_steps: int, slices=(1.0, 2.0, 4.0, 8.0), max_lane_sms: int = 32,
                 load_factor: float = 1.2, solo: int = 0):
        self.ens = ens
        self.max_steps = int(max_steps)
        self.slices = [float(s) for s in slices]
        self.max_lane_sms = int(max_lane_sms)
        self.load_factor = float(load_factor)
        self.solo = int(solo)
        self.history: List[dict] = []
        import torch
        self.sm_count = torch.cuda.get_device_properties(ens.device).multi_processor_count

    def plan(self, K, t_end, t0, a0, t, attempts, active) -> WorkList:
        wl, info = adaptive_work_list(K, t_end, t0, a0, t, attempts, active, self.sm_count, self.max_lane_sms,
                                      self.load_factor, self.MIN_OBSERVED, self.solo)
        self.history.append(info)
        return wl

    def launch(self, stream=None) -> None:
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.ens.device)
        with torch.cuda.stream(st):   # reads, timing events and solves all on one stream
            self._launch(st)

    def _launch(self, stream) -> None:
        import torch
        ens, d = self.ens, self.ens.dev
        K = ens.host["K"]
        t_end = d["t_end"].cpu().numpy()
        t0 = d["t"].cpu().numpy()
        a0 = (d["steps"] + d["rejected"]).cpu().numpy().astype(np.int64)
        self.history = []
        for sl in self.slices + [0.0]:
            t = d["t"].cpu().numpy()
            status = d["status"].cpu().numpy()
            steps = d["steps"].cpu().numpy()
            attempts = steps.astype(np.int64) + d["rejected"].cpu().numpy()
            active = ((status == _lib.ACTIVE) | (status == _lib.MAX_STEPS_REACHED)) & (steps < self.max_steps)
            if not np.any(active):
                break
            wl = self.plan(K, t_end, t0, a0, t, attempts, active)
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
            ens.solve(self.max_steps, work=wl, stream=stream, budget_ns=int(sl * 1e9), steps_total=True)
            ev[1].record()
            torch.cuda.synchronize(ens.device)
            self.history[-1].update(slice_s=sl, device_s=ev[0].elapsed_time(ev[1]) * 1e-3,
                                    attempts_before=int(attempts.sum() - a0.sum()))

    def close(self) -> None:
        pass


class Plan:
    """A captured CUDA graph of one batched solve bound to an ensemble's
    device arrays.  ``launch()`` replays it (a single graph launch)."""

    def __init__(self, ens: Ensemble, max_steps: int, work: Optional[WorkList]):
        self.ens = ens
        self.ctx = _lib.default_context(ens.device)
        self._spec, self._e = ens.spec(), ens.abi()
        self._w, self._keep = ens.work(work)
        import torch
        torch.cuda.synchronize(ens.device)   # the order upload is complete before any replay, on any stream
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
