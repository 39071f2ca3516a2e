"""Continuous-batching solve server on one GPU, device-resident.

Requests (one CKM1D system each: K bubbles, radii, drive, positions, span)
arrive at any time.  The server owns one preallocated ragged ensemble on the
device -- a table of system slots, a pool of bubble rows and a pool of
coupling storage -- and runs a loop of ticks:

  1. admit   -- queued requests, oldest first, are admitted while the pools
                have room for them: a free slot, K contiguous bubble rows and
                3 K^2 coupling elements (admission by device memory, any K
                <= 32 in one pool).  The host only packs the raw requests into
                a pinned staging buffer; one host->device copy, then the
                parameter precompute and the initial state are written on the
                GPU (cbc_admit, bit-identical to the host precompute);
  2. advance -- one batched solve over every occupied slot for a slice of
                device time (cbc_work.budget_ns): each warp steps its systems
                until the slice ends, then stops them after their current step
                (status -1, resumable bit for bit).  Oldest requests are
                claimed first.  max_steps caps the steps a request accumulates
                over all slices;
  3. harvest -- the status and step counters of the slot table come back in
                one asynchronous copy into pinned memory (8 bytes per slot);
                finished requests release their slot and pool ranges.

State never leaves the GPU between slices; the host sees only statuses and,
on request, the results of finished requests.  A request's result does not
depend on what else is in flight (alone == in the mix, tests/test_serving.py).
Latency = the end of the tick that saw the request finish - its arrival.
No reference counterpart: the reference only runs fixed batches through
Model.solve (models/model.py:108-162); the per-system integration is the same
kernel and arithmetic as every other path.
"""
from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from . import _lib, admission, scenes
from .admission import RangeAllocator
from .ensemble import cost_weight
from .models import SolverSpec, water


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
    admitted: float = -1.0
    done: float = -1.0
    slot: int = -1
    status: int = 0
    result: Optional[Dict[str, np.ndarray]] = None


# device bytes a request of K bubbles occupies in the pools (state + bubble
# constants per bubble, coupling block, per-system rows and scalars)
def request_bytes(K: int, nk: int = 2) -> int:
    return 160 * K + 24 * K * K + (8 * 8 + 8 * 4 * nk + 8 * 7 + 4 * 6)


class SolveServer:
    """Device-resident continuous batching over one slot table.

    max_systems: slot-table size (requests in flight at most);
    memory_bytes: device memory for the bubble-row and coupling pools
    (default: enough for every slot to hold K = 16); slice_ms: device time
    per advance.  ``slots`` (a dict K -> count) is accepted for callers of the
    earlier per-bucket interface and only sizes the pools.
    """

    def __init__(self, slots: Optional[Dict[int, int]] = None, max_systems: int = 0, memory_bytes: int = 0,
                 nk: int = 2, ac: str = "SW_A", freqs_khz=(25.0, 50.0), ref_freq_khz: float = 25.0,
                 slice_ms: float = 2.0, chunk_steps: int = 0, max_steps: int = 1_000_000,
                 solver_spec: Optional[SolverSpec] = None, device: int = 0, keep_results: bool = False):
        import torch
        self.nk, self.ac, self.freqs = int(nk), ac, tuple(float(f) for f in freqs_khz)
        self.max_steps = int(max_steps)
        self.slice_ns = int(slice_ms * 1e6)
        self.chunk_steps = int(chunk_steps)        # > 0: a step budget per advance instead of a time slice
        self.keep_results = keep_results
        self.device = device
        self.solver_spec = solver_spec if solver_spec is not None else SolverSpec()
        dev = torch.device("cuda", device)
        if slots:
            max_systems = max_systems or int(sum(slots.values()))
            rows = int(sum(k * n for k, n in slots.items()))
            coup = int(sum(3 * k * k * n for k, n in slots.items()))
        else:
            max_systems = max_systems or 16384
            per = memory_bytes // max_systems if memory_bytes else 0
            kcap = 16
            if per:
                while kcap > 1 and 160 * kcap + 24 * kcap * kcap > per:
                    kcap //= 2
            rows, coup = max_systems * kcap, max_systems * 3 * kcap * kcap
        self.S = int(max_systems)
        f64, i32, i64 = torch.float64, torch.int32, torch.int64
        z = lambda n, dt: torch.zeros(n, dtype=dt, device=dev)   # noqa: E731
        self.d = {
            "bubble_offset": z(self.S, i64), "coupling_offset": z(self.S, i64),
            "state": z((rows, 4), f64), "unit_params": z((rows, 16), f64),
            "system_params": z((self.S, 8), f64), "control_params": z((self.S, 4 * self.nk), f64),
            "coupling": z(max(coup, 1), f64), "t": z(self.S, f64), "t_end": z(self.S, f64),
            "t_begin": z(self.S, f64), "h": z(self.S, f64), "event": z(self.S, f64),
            "status": torch.ones(self.S, dtype=i32, device=dev), "steps": z(self.S, i32),
            "rejected": z(self.S, i32), "conv_ok": z(self.S, i32), "conv_fail": z(self.S, i32),
            "lin_iters": z(self.S, i64),
        }
        self.rows = RangeAllocator(rows)
        self.coup = RangeAllocator(coup)
        self.free_slots = deque(range(self.S))
        self.slot_K = np.zeros(self.S, np.int32)
        # tick at which the slot's current request was admitted (-1: free);
        # a read-back taken at an earlier tick says nothing about it
        self.slot_tick = np.full(self.S, -1, np.int64)
        self.busy: Dict[int, Request] = {}
        self.busy_order = np.zeros(0, np.int32)     # occupied slots in admission order
        self.queue: deque = deque()
        self.completed: List[Request] = []
        self.stream = torch.cuda.Stream(device=dev)
        # pinned staging: request records, the work list, the status read-back
        # (two of each: the host fills one while the GPU may still read the other)
        self.rl = _lib.admit_record_len(self.nk)
        self.rec_cap = 4096
        self.h_rec = [torch.zeros((self.rec_cap, self.rl), dtype=f64).pin_memory() for _ in range(2)]
        self.d_rec = [torch.zeros((self.rec_cap, self.rl), dtype=f64, device=dev) for _ in range(2)]
        self.d_order = [torch.zeros(self.S, dtype=i32, device=dev) for _ in range(2)]
        self.h_order = [torch.zeros(self.S, dtype=i32).pin_memory() for _ in range(2)]
        self.h_status = [torch.zeros(self.S, dtype=i32).pin_memory() for _ in range(2)]
        self.h_steps = [torch.zeros(self.S, dtype=i32).pin_memory() for _ in range(2)]
        self.readback = [None, None]             # (event, slots advanced) per buffer
        self.pipelined = True
        self.consts = admission.consts_struct(water(), ref_freq_khz)
        self.ctx = _lib.default_context(device)
        self.lib = _lib.lib()
        self.abi = self._abi()
        self.spec = self._spec()
        self.ticks = 0
        torch.cuda.synchronize(device)     # the pools are initialised before the server stream uses them
        self.t0 = time.perf_counter()

    # ---- ABI structures (built once; the arrays never move) ----
    def _abi(self) -> _lib.cbc_ensemble:
        d = self.d
        e = _lib.cbc_ensemble()
        e.ns, e.nb = self.S, int(d["state"].shape[0])
        e.up_stride, e.sp_stride, e.cp_stride = 16, 8, 4 * self.nk
        for name in ("bubble_offset", "coupling_offset", "state", "unit_params", "system_params",
                     "control_params", "coupling", "t", "t_end", "t_begin", "h", "event", "status",
                     "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
            setattr(e, name, d[name].data_ptr())
        return e

    def _spec(self) -> _lib.cbc_spec:
        s = self.solver_spec
        return _lib.cbc_spec(self.S, 0, 0, 0, self.nk, _lib.AC_CODES[self.ac], _lib.DENSE_CODES[s.dense_mode],
                             int(s.lin_max_iter), s.atol, s.rtol, s.min_step, s.max_step, s.lin_atol, s.lin_rtol,
                             s.lin_relaxation, s.etol, s.col_threshold, _lib.LIN_CODES[s.lin_solver], 0)

    def now(self) -> float:
        return time.perf_counter() - self.t0

    # ---- client side ----
    def submit(self, req: Request) -> None:
        if not 1 <= req.K <= 32:
            raise ValueError(f"K = {req.K}: 1..32 bubbles per request")
        if len(req.PA) != self.nk or len(req.PS) != self.nk:
            raise ValueError(f"PA and PS need {self.nk} harmonic components")
        self.queue.append(req)

    # ---- loop ----
    def _admit(self) -> int:
        import torch
        took: List[Request] = []
        offs = []
        while self.queue and self.free_slots and len(took) < self.rec_cap:
            r = self.queue[0]
            b = self.rows.alloc(r.K)
            if b is None:
                break
            c = self.coup.alloc(3 * r.K * r.K)
            if c is None:
                self.rows.free(b, r.K)
                break                               # oldest first: no overtaking
            self.queue.popleft()
            s = self.free_slots.popleft()
            took.append(r)
            offs.append((s, b, c))
        if not took:
            return 0
        n = len(took)
        par = self.ticks & 1
        rec = self.h_rec[par].numpy()
        admission.pack_records([r.K for r in took], [o[0] for o in offs], [o[1] for o in offs],
                               [o[2] for o in offs], [r.span for r in took],
                               np.stack([r.PA for r in took]), np.tile(np.asarray(self.freqs), (n, 1)),
                               np.stack([r.PS for r in took]), [r.R0 for r in took], [r.X0 for r in took], out=rec)
        t = self.now()
        with torch.cuda.stream(self.stream):
            self.d_rec[par][:n].copy_(self.h_rec[par][:n], non_blocking=True)
        self.ctx.check(self.lib.cbc_admit(self.ctx.handle, ctypes.byref(self.abi), ctypes.byref(self.consts),
                                          self.d_rec[par].data_ptr(), n, self.nk,
                                          int(self.d["coupling"].numel()),
                                          ctypes.c_void_p(self.stream.cuda_stream)))
        for r, (s, b, c) in zip(took, offs):
            r.slot, r.admitted = s, t
            r._ranges = (b, c)
            self.slot_K[s] = r.K
            self.slot_tick[s] = self.ticks
            self.busy[s] = r
        self.busy_order = np.concatenate([self.busy_order, np.asarray([o[0] for o in offs], np.int32)])
        return n

    def _advance(self) -> None:
        import torch
        if self.busy_order.size == 0:
            return
        slots = self.busy_order
        K = self.slot_K[slots]
        ks = np.unique(K)[::-1]
        order, begins = [], [0]
        for k in ks:
            sel = slots[K == k]                     # admission order inside the bucket
            order.append(sel)
            begins.append(begins[-1] + sel.size)
        o = np.concatenate(order)
        par = self.ticks & 1
        self.h_order[par].numpy()[:o.size] = o
        with torch.cuda.stream(self.stream):
            self.d_order[par][:o.size].copy_(self.h_order[par][:o.size], non_blocking=True)
        bk = np.ascontiguousarray(ks, np.int32)
        bb = np.asarray(begins, np.int32)
        w = _lib.cbc_work()
        w.order = self.d_order[par].data_ptr()
        w.nbuckets = int(bk.size)
        w.bucket_K = bk.ctypes.data
        w.bucket_begin = bb.ctypes.data
        # every bucket starts with a share of the GPU proportional to the cost
        # of one step of all its systems: without shares each bucket's grid
        # asks for the whole GPU, and whichever kernel's blocks reach the SMs
        # first holds them for the slice
        sh = None
        if bk.size > 1:
            c = np.diff(bb).astype(np.float64) * cost_weight(bk)
            sh = (c / c.sum()).astype(np.float32)
            w.share = sh.ctypes.data
        if self.chunk_steps > 0:
            max_steps, w.steps_total = self.chunk_steps, 0
        else:
            max_steps, w.steps_total, w.budget_ns = self.max_steps, 1, self.slice_ns
        self.ctx.check(self.lib.cbc_ensemble_solve(self.ctx.handle, ctypes.byref(self.spec), ctypes.byref(self.abi),
                                                   ctypes.byref(w), int(max_steps),
                                                   ctypes.c_void_p(self.stream.cuda_stream)))

    def _readback(self) -> None:
        """Enqueues the copy of the slot table's statuses and step counters
        into this tick's pinned buffers (after the tick's solve)."""
        import torch
        par = self.ticks & 1
        if self.busy_order.size == 0:
            self.readback[par] = None
            return
        with torch.cuda.stream(self.stream):
            self.h_status[par].copy_(self.d["status"], non_blocking=True)
            self.h_steps[par].copy_(self.d["steps"], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.readback[par] = (ev, self.busy_order.copy(), self.ticks)

    def _harvest(self, par: int) -> int:
        """Releases the requests that had finished by the read-back `par`."""
        rb = self.readback[par]
        if rb is None:
            return 0
        ev, slots, tick = rb
        self.readback[par] = None
        ev.synchronize()
        # only requests admitted no later than the read-back's tick and not
        # released since (a slot may have been released by the other
        # read-back and refilled after this one was taken)
        slots = slots[(self.slot_tick[slots] >= 0) & (self.slot_tick[slots] <= tick)]
        if slots.size == 0:
            return 0
        st = self.h_status[par].numpy()
        steps = self.h_steps[par].numpy()
        s_st, s_steps = st[slots], steps[slots]
        # 0: not yet claimed; -1: stopped by the slice; else finished.  A
        # step-budget chunk (chunk_steps) ends a request only at its own cap.
        fin = (s_st != 0) & (s_st != -1) | (s_steps >= self.max_steps)
        if not np.any(fin):
            return 0
        tnow = self.now()
        done = slots[fin]
        if self.keep_results:
            self.stream.synchronize()            # results read after the slice in flight
        for s in done:
            r = self.busy.pop(int(s))
            r.done = tnow
            r.status = int(st[s])
            if self.keep_results:
                r.result = self.result_of(int(s))
            b, c = r._ranges
            self.rows.free(b, r.K)
            self.coup.free(c, 3 * r.K * r.K)
            self.slot_tick[s] = -1
            self.free_slots.append(int(s))
            self.completed.append(r)
        self.busy_order = self.busy_order[~np.isin(self.busy_order, done)]
        return int(done.size)

    def result_of(self, slot: int) -> Dict[str, np.ndarray]:
        r = self.busy.get(slot)
        k = int(self.slot_K[slot])
        b0 = int(self.d["bubble_offset"][slot].item())
        d = self.d
        return {"state": d["state"][b0:b0 + k].cpu().numpy(), "t": float(d["t"][slot]),
                "status": int(d["status"][slot]), "steps": int(d["steps"][slot]), "h": float(d["h"][slot])}

    def step(self) -> int:
        """One admit / advance / read-back tick; returns completions.

        Pipelined: the tick enqueues its solve and status read-back, then
        harvests the previous tick's read-back while the GPU works on this
        one, so the host's bookkeeping overlaps the device time.  A request
        is therefore released one tick after the slice that finished it
        (its slot idles through that slice; results are unaffected)."""
        self._admit()
        self._advance()
        self._readback()
        par = self.ticks & 1
        self.ticks += 1
        if self.pipelined:
            return self._harvest(par ^ 1)
        return self._harvest(par)

    def drain(self) -> int:
        """Harvests every outstanding read-back."""
        return self._harvest(0) + self._harvest(1)

    def advanced_system_periods(self) -> float:
        """Simulated time advanced so far by every request in flight or done."""
        done = sum(r.span if r.status == 1 else 0.0 for r in self.completed)
        if self.busy_order.size == 0:
            return done
        t = self.d["t"].cpu().numpy()
        return done + float(np.sum(t[self.busy_order]))

    def idle(self) -> bool:
        return not self.busy and not self.queue and self.readback[0] is None and self.readback[1] is None

    def occupancy(self) -> Dict[str, float]:
        return {"systems": len(self.busy), "rows_used": self.rows.used, "coupling_used": self.coup.used,
                "queued": len(self.queue)}


def latency_stats(done: List[Request]) -> Dict[str, float]:
    lat = np.asarray([r.done - r.arrival for r in done])
    if lat.size == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p95_ms": float(np.percentile(lat, 95) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "completed": int(lat.size)}


def requests_from_scene(scene: scenes.Scene, arrivals: np.ndarray) -> List[Request]:
    """Requests of a (ragged) scene with the given arrival times (s)."""
    return [Request(rid=i, K=int(scene.K[i]), R0=np.asarray(scene.R0[i]), PA=scene.PA[:, i].copy(),
                    PS=scene.PS[:, i].copy(), X0=np.asarray(scene.X0[i]), span=float(scene.t_end[i]),
                    arrival=float(arrivals[i])) for i in range(scene.ns)]


def serve_stream(server: SolveServer, reqs: List[Request], duration_s: float, drain: bool = False) -> Dict:
    """Plays an arrival-time-stamped request stream against the server's
    clock for `duration_s` seconds (then drains if asked) and reports latency
    percentiles of the completed requests and the achieved throughput
    against the offered load."""
    pending = deque(sorted(reqs, key=lambda r: r.arrival))
    server.t0 = time.perf_counter()
    offered = sum(r.span for r in reqs if r.arrival < duration_s)
    while True:
        t = server.now()
        while pending and pending[0].arrival <= t:
            server.submit(pending.popleft())
        server.step()
        if t >= duration_s and (not drain or server.idle()):
            break
        if not pending and server.idle():
            break
    server.drain()
    wall = server.now()
    done = server.completed
    adv = sum(r.span for r in done if r.status == 1)
    advanced = server.advanced_system_periods()
    out = latency_stats(done)
    out.update({"duration_s": duration_s, "wall_s": wall, "submitted": sum(1 for r in reqs if r.arrival < duration_s),
                "completed": len(done), "in_flight": len(server.busy), "queued": len(server.queue),
                "offered_system_periods_per_s": offered / duration_s,
                "completed_system_periods_per_s": adv / wall,
                "advanced_system_periods_per_s": advanced / wall, "ticks": server.ticks})
    return out
