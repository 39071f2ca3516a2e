"""Benchmark of the CKM1D ensemble integrator on B200.

Metric (system-periods/s at rtol = atol = 1e-9): one system-period is one
coupled-bubble system advanced by one period of the 25 kHz reference drive.
Workload at N=1: the mixed-K batched ensemble -- 65,536 systems, K in
{2,3,4,6,8} (p .4/.2/.2/.1/.1), spans U[5,50] periods, water, dual-frequency
standing wave (25 + 50 kHz), FP64, seeded synthetic inputs (no dataset exists).
A step is one batched solve of the whole ensemble starting from the same
initial state: the adaptive schedule (the persistent work-stealing kernels
in device-time slices, the host re-planning buckets and latency lanes between
slices; `--schedule span` makes it one CUDA-graph launch).

Also measured in the 1-GPU job (outside the timed steps): the plain
one-launch-per-K reference-layout path on the same ensemble (the reference's
execution model: one (NS, K) kernel per K, relaunched every 2048 steps with a
host check), the direct coupling solve, the vec-env step latency, the served
streams, the large-K dense output, the plain parameter study and the CPU
oracle.  `--workload alone | large_k | served | costs` runs one of them alone.

Multi-GPU (torchrun): weak scaling, every rank solves its own 65,536-system
ensemble (seed + rank); no collective on the data path, only the final
max-time / sum-work reduction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "coupled-bubble-control_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "system-periods/s @rtol 1e-9, batched vs plain; p50/p99 env-step latency"
# DRAM traffic of the dominant kernel per launch (ncu, see roofline.traffic_note)
TRAFFIC_K8_BYTES = 20219904    # 20,158,720 read + 61,184 written
UNIT = "system-periods/s"
MAX_STEPS = 1_000_000


def status_counts_by_k(K, status):
    """{K: {status: count}} of a finished solve."""
    out = {}
    for k in np.unique(K):
        sel = np.asarray(K) == k
        out[f"K{int(k)}"] = {int(a): int(b) for a, b in zip(*np.unique(np.asarray(status)[sel], return_counts=True))}
    return out


def lu_flops(K):
    """Flops of one direct solve (Gauss-Jordan with partial pivoting) of the
    N = 2K coupling system: N^2 (N + 1) multiply-adds (fma = 2) over every row
    and column, N^2 multipliers, N reciprocals, N products for x, and the
    2K(K - 1) cpf0 scalings of the matrix rows."""
    K = np.asarray(K, dtype=np.float64)
    N = 2.0 * K
    return N * N * (N + 1.0) + N * N + 2.0 * N + 2.0 * K * (K - 1.0)


def flop_count(K, steps, lin_iters, lin_solver="richardson"):
    """Algorithmic FP64 flops (add/mul = 1, fma = 2, div/sqrt/pow/sin/cos = 1):
    per step 6 RHS of 130K + 35K^2 (uncoupled RHS + explicit coupling) plus
    240K + 10 (stages, error norm, controller), plus 20K^2 + 12K per
    Richardson sweep of the implicit coupling, or lu_flops(K) per direct
    solve (lin_iters counts sweeps, or solves)."""
    K = np.asarray(K, dtype=np.float64)
    steps = np.asarray(steps, dtype=np.float64)
    lin = np.asarray(lin_iters, dtype=np.float64)
    per_step = 6.0 * (130.0 * K + 35.0 * K ** 2) + 240.0 * K + 10.0
    per_lin = lu_flops(K) if lin_solver == "lu" else 20.0 * K ** 2 + 12.0 * K
    return float(np.sum(steps * per_step + lin * per_lin))


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons every 200 ms while active."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def job_totals(rank_ms: float, rank_work: float, dist=None, device=None):
    """Whole-job figures: the slowest rank's time and the work of all ranks.
    Every rank must call this (it is a collective when ``dist`` is given)."""
    if dist is None:
        return rank_ms, rank_work
    import torch
    t = torch.tensor([rank_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w = torch.tensor([rank_work], dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def rank_seed(rank: int) -> int:
    """Each replica integrates its own ensemble (weak scaling)."""
    return 1 + rank


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_fp64_peak(dev) -> float:
    """cuBLAS FP64 GEMM throughput (TFLOP/s), best of 5: the measured FP64
    denominator of the roofline (the driver's peaks file covers HBM and bf16)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def cpu_baseline(scene, seconds: float = 12.0, nthreads: int = 0, seed: int = 99, step_cap: int = 300_000):
    """The CPU oracle (C++ restatement of the reference integrator) on every
    host core over a bounded random sample of the same workload: one worker
    thread per core pulls systems in a random order, one system per oracle
    call, each integrated over its FULL span (at most `step_cap` steps),
    until `seconds` have passed; the systems in flight then finish.  The
    rate is the system-periods advanced over the busy time per core (the
    throughput of the cores kept busy, as a long run over the whole ensemble
    keeps them); the wall-clock rate of the sample, tail included, is in
    `sample`."""
    import threading
    from concurrent.futures import ThreadPoolExecutor
    from cbc_b200 import scenes
    from oracle import oracle
    cores = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    perm = np.random.default_rng(seed).permutation(scene.ns)
    lock = threading.Lock()
    st = {"pos": 0, "adv": 0.0, "busy": 0.0, "done": 0, "capped": 0}
    t0 = time.perf_counter()

    def worker():
        while True:
            with lock:
                if time.perf_counter() - t0 >= seconds or st["pos"] >= scene.ns:
                    return
                i = int(perm[st["pos"]])
                st["pos"] += 1
            a = time.perf_counter()
            m = scenes.build_model(scenes.subset(scene, np.array([i])), ndo=0)
            buf = oracle.solve_model(m, max_steps=step_cap, kernel_steps=step_cap, nthreads=1)
            b = time.perf_counter()
            with lock:
                st["adv"] += float(np.sum(buf["actual_time"]))
                st["capped"] += int(np.sum(buf["status_flags"] == -1))
                st["busy"] += b - a
                st["done"] += 1

    with ThreadPoolExecutor(cores) as ex:
        for f in [ex.submit(worker) for _ in range(cores)]:
            f.result()
    wall = time.perf_counter() - t0
    value = st["adv"] / (st["busy"] / cores)
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{st['done']} systems drawn at random from the same mixed-K ensemble, each over its full "
                      f"5-50 period span ({st['capped']} stopped at the {step_cap}-step cap), "
                      f"{st['adv']:.1f} system-periods, CPU oracle (C++ restatement of the reference integrator) "
                      f"on {cores} threads, one system per thread at a time; {st['busy']:.1f} thread-seconds "
                      f"busy in {wall:.1f} s of wall time ({st['adv'] / wall:.1f} system-periods/s by wall "
                      f"clock, the tail of the last systems included)"}


def workload_config(args, world: int) -> dict:
    """The workload both arms report (the reference arm times a bounded CPU
    sample of it, described in its cpu_baseline.sample)."""
    wname = f"mixed_k_{args.ns}" + (f"_only_K{args.only_k}" if args.only_k > 0 else "")
    return {"workload": wname, "ns_per_gpu": args.ns, "K": [2, 3, 4, 6, 8],
            "K_weights": [0.4, 0.2, 0.2, 0.1, 0.1], "span_periods": [5, 50], "rtol": 1e-9,
            "atol": 1e-9, "max_steps": args.max_steps, "field": "SW_A 25+50 kHz", "lin_solver": args.lin_solver,
            "l2": "256 MiB buffer written before every step", "parallelism": f"replicas{world}",
            "schedule": args.schedule}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from cbc_b200 import scenes
    scene = scenes.mixed_k(ns=args.ns, seed=1)
    # each step is a bounded sample; many steps get smaller samples so that
    # the whole run stays within a few minutes
    nstep = max(1, args.warmup + args.steps)
    sec = min(12.0, max(3.0, 120.0 / nstep))
    vals = []
    for i in range(nstep):
        r = cpu_baseline(scene, seconds=sec, seed=99 + i)
        if i >= args.warmup:
            vals.append(r["value"])
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, world),
            "cpu_baseline": {**r, "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


ADAPTIVE_OPTS = {}   # slices / load_factor of the adaptive schedule (command line)


def make_plan(ens, schedule: str, max_steps: int = MAX_STEPS):
    """adaptive: time slices with re-planning and latency lanes; pilot: one
    measured re-ordering after a short pilot pass; span: longest span first."""
    if schedule == "adaptive":
        return ens.adaptive_plan(max_steps, **ADAPTIVE_OPTS)
    if schedule == "pilot":
        return ens.scheduled_plan(max_steps, pilot_steps=min(256, max_steps - 1))
    return ens.plan(max_steps)


def batched_once(scene, dev_index: int, schedule: str) -> float:
    """System-periods/s of one batched solve of `scene` (for the ratio)."""
    import torch
    from cbc_b200.ensemble import Ensemble
    ens = Ensemble.from_scene(scene, device=dev_index).to_device()
    plan = make_plan(ens, schedule)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan.launch()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    adv = float((ens.dev["t"] - torch.from_numpy(ens.host["t"]).to(ens.dev["t"].device)).sum().item())
    plan.close()
    return adv / dt


def plain_study_measure(dev_index: int, cpu_systems: int = 64):
    """The plain parameter study (1,024 systems of K = 2, 10 periods, 32
    samples per period, seed 0) through the reference drop-in path
    (Model.solve: reference-layout buffers, relaunch every 2,048 steps with a
    host completion check), and the CPU oracle on `cpu_systems` of them on
    every host core."""
    import torch
    from cbc_b200 import scenes
    from oracle import oracle
    sc = scenes.plain_study(ns=1024, periods=10.0, samples_per_period=32, seed=0)
    m = scenes.build_model(sc)
    m._ensure_buffers()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m.solve(max_steps=MAX_STEPS, kernel_steps=2048)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    adv = float(m.runtime.device_buffers.state.actual_time.sum().item())
    sub = scenes.subset(sc, np.arange(cpu_systems))
    mc = scenes.build_model(sub)
    t1 = time.perf_counter()
    buf = oracle.solve_model(mc, max_steps=MAX_STEPS, kernel_steps=2048)
    cdt = time.perf_counter() - t1
    cadv = float(np.sum(buf["actual_time"]))
    return {"workload": "plain_study_1024xK2_10periods_321samples", "value": adv / dt, "unit": UNIT,
            "seconds": dt, "path": "Model.solve (reference layout, relaunch every 2048 steps)",
            "cpu_oracle": {"value": cadv / cdt, "unit": UNIT, "systems": cpu_systems,
                           "cores": os.cpu_count() or 1},
            "gpu_vs_cpu": (adv / dt) / (cadv / cdt)}


def plain_per_k(scene, dev, solver_spec=None):
    """The reference execution model on the same systems: one reference-layout
    solve per K (cbc_solve, relaunch every 2048 steps with a host check)."""
    import torch
    from cbc_b200 import scenes
    total = 0.0
    adv = 0.0
    for k in np.unique(scene.K):
        sel = np.nonzero(scene.K == k)[0]
        m = scenes.build_model(scenes.subset(scene, sel), ndo=0, solver_spec=solver_spec)
        m._ensure_buffers()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.solve(max_steps=MAX_STEPS, kernel_steps=2048)
        torch.cuda.synchronize()
        total += time.perf_counter() - t0
        adv += float(m.runtime.device_buffers.state.actual_time.sum().item())
    return adv / total, total


def alone_latency(scene, dev_index: int, lin_solver: str, attempts: int = 3000, ks=(2, 4, 8)):
    """Per-attempt latency (us) of single systems running alone (one warp on
    an otherwise idle GPU): for each K in `ks`, the longest-span system of
    that K in the workload, `attempts` step attempts from its initial state."""
    import torch
    from cbc_b200 import scenes
    from cbc_b200.ensemble import Ensemble
    from cbc_b200.models import SolverSpec
    out = {}
    for k in ks:
        sel = np.nonzero(scene.K == k)[0]
        if sel.size == 0:
            continue
        s = int(sel[np.argmax(scene.t_end[sel])])
        ens = Ensemble.from_scene(scenes.subset(scene, [s]), solver_spec=SolverSpec(lin_solver=lin_solver),
                                  device=dev_index).to_device()
        ens.solve(50)                      # load the kernel
        ens.reset_device()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ens.solve(attempts)
        b.record()
        torch.cuda.synchronize()
        n = int((ens.dev["steps"] + ens.dev["rejected"]).sum().item())
        out[f"K{k}_us_per_attempt"] = a.elapsed_time(b) * 1e3 / max(n, 1)
    return out


def lu_arm(scene, dev_index: int, schedule: str, flush, max_steps: int = MAX_STEPS, plain: bool = True,
           tune: bool = True):
    """The same workload with the direct coupling solve (lin_solver = "lu"):
    one untimed and one timed batched solve (L2 flushed before), its status
    counts and roofline numerator, and optionally the plain per-K path."""
    import torch
    from cbc_b200.ensemble import Ensemble
    from cbc_b200.models import SolverSpec
    spec = SolverSpec(lin_solver="lu")
    ens = Ensemble.from_scene(scene, solver_spec=spec, device=dev_index).to_device()
    tune_info = None
    if tune:
        from cbc_b200.autotune import Autotuner
        tuner = Autotuner(dev_index)
        tuner.tune(ens)
        tune_info = tuner.summary()
    plan = make_plan(ens, schedule, max_steps)
    pristine = {k: v.clone() for k, v in ens.dev.items()}
    ms = None
    for i in range(2):
        for k in ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
            ens.dev[k].copy_(pristine[k])
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.launch()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
    plan.close()
    res = ens.to_host()
    adv = float(np.sum(res["t"] - ens.host["t"]))
    flops = flop_count(res["K"], res["steps"], res["lin_iters"], "lu")
    out = {"value": adv / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "advanced_system_periods_per_step": adv,
           "status_counts": {int(k): int(v) for k, v in zip(*np.unique(res["status"], return_counts=True))},
           "status_counts_by_K": status_counts_by_k(res["K"], res["status"]),
           "steps_per_solve": int(np.sum(res["steps"])), "algorithmic_gflop_per_step": flops / 1e9,
           "achieved_tflops": flops / (ms * 1e-3) / 1e12, "autotune": tune_info}
    if plain:
        pv, ptime = plain_per_k(scene, None, spec)
        out["plain"] = {"value": pv, "unit": UNIT, "seconds": ptime}
        out["batched_vs_plain"] = out["value"] / pv
    return out


def env_step_latency(dev_index: int, n_steps: int = 128, warmup: int = 3, envs_per_warp: int = -1):
    """PPO vec-env stepping: 1024 envs x K=4 bubbles (R0 60 um, SW_N, 25+50 kHz),
    5 periods per env step, actions (PA_1, PA_2) ~ U[0, 1.5] bar from seed 2,
    float32 observation written in place, 128-step horizon with resets.
    Returns p50/p95/p99 of the env-step time measured with CUDA events."""
    import torch
    from cbc_b200.envs import CKM1DVecEnv
    kw = {} if envs_per_warp < 0 else {"envs_per_warp": envs_per_warp}
    env = CKM1DVecEnv(num_envs=1024, num_bubbles=4, time_step_length=5.0, episode_length=128, seed=42,
                      device=dev_index, **kw)
    env.reset()
    gen = torch.Generator(device=torch.device("cuda", dev_index)).manual_seed(2)
    times = []
    for i in range(warmup + n_steps):
        act = torch.rand((1024, 2), device=torch.device("cuda", dev_index), generator=gen) * 1.5
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        env.step(act)
        b.record()
        b.synchronize()
        if i >= warmup:
            times.append(a.elapsed_time(b))
    env.close()
    t = np.asarray(times)
    return {"p50_ms": float(np.percentile(t, 50)), "p95_ms": float(np.percentile(t, 95)),
            "p99_ms": float(np.percentile(t, 99)), "mean_ms": float(t.mean()), "steps": int(t.size),
            "envs": 1024, "K": 4, "periods_per_step": 5.0,
            "env_system_periods_per_s": float(1024 * 5.0 / (t.mean() * 1e-3))}


def large_k_measure(dev_index: int, ns: int = 16384, periods: float = 0.5, peak_tflops: float = 0.0):
    """Large-K dense output (K = 32, one warp per system, 64 samples per
    period): one batched solve of `ns` systems over `periods` periods from
    resident inputs.  Reports system-periods/s, the FP64 roofline numerator
    and the HBM rate of the trajectory writes (dense samples + times)."""
    import torch
    from cbc_b200 import scenes
    from cbc_b200.ensemble import Ensemble
    sc = scenes.large_k(ns=ns, K=32, periods=periods, samples_per_period=64, seed=4)
    ens = Ensemble.from_scene(sc, device=dev_index).to_device()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ens.solve(MAX_STEPS)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    res = ens.to_host()
    adv = float(np.sum(res["t"] - ens.host["t"]))
    samples = int(np.sum(res["dense_index"]))
    dense_bytes = samples * 32 * 4 * 8 + samples * 8
    flops = flop_count(res["K"], res["steps"], res["lin_iters"])
    out = {"workload": f"large_k_{ns}x32_{periods:g}periods_64spp", "systems": ns, "K": 32,
           "periods": periods, "dense_samples": int(sc.ndo), "value": adv / (ms * 1e-3), "unit": UNIT,
           "ms": ms, "status_counts": {int(k): int(v) for k, v in zip(*np.unique(res["status"], return_counts=True))},
           "trajectory_bytes": dense_bytes, "trajectory_hbm_gbs": dense_bytes / (ms * 1e-3) / 1e9,
           "bytes_per_system_period": dense_bytes / max(adv, 1e-30),
           "achieved_tflops": flops / (ms * 1e-3) / 1e12,
           "note": "span reduced from 200 to %g periods: 200 periods of 16,384 systems write 216 GB of "
                   "samples (more than the GPU holds) and take hours of FP64 work" % periods}
    if peak_tflops > 0:
        out["roofline_frac"] = out["achieved_tflops"] / peak_tflops
    return out


def served_measure(dev_index: int, rate_hz: float, duration_s: float, seed: int = 3):
    """Served solve stream: Poisson arrivals at `rate_hz`, K ~ U{2,4,8,16},
    spans U[1,50] periods, played for `duration_s` seconds against the
    device-resident server (requests admitted by free pool memory)."""
    from cbc_b200 import scenes
    from cbc_b200.serving import SolveServer, requests_from_scene, serve_stream
    n = int(rate_hz * duration_s * 1.2) + 16
    arrivals, sc = scenes.served_stream(duration_s=duration_s, rate_hz=rate_hz, seed=seed, max_requests=n)
    reqs = requests_from_scene(sc, arrivals)
    srv = SolveServer(max_systems=65536, memory_bytes=2 << 30, slice_ms=2.0, device=dev_index)
    out = serve_stream(srv, reqs, duration_s)
    out.update({"rate_hz": rate_hz, "K": [2, 4, 8, 16], "span_periods": [1, 50]})
    return out


def run_b200(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    from cbc_b200 import scenes, _lib
    from cbc_b200.ensemble import Ensemble

    scene = scenes.mixed_k(ns=args.ns, seed=rank_seed(rank))
    if args.only_k > 0:      # profiling cases: one K bucket of the workload, filling the GPU
        scene = scenes.subset(scene, np.nonzero(scene.K == args.only_k)[0])
    from cbc_b200.models import SolverSpec
    ens = Ensemble.from_scene(scene, solver_spec=SolverSpec(lin_solver=args.lin_solver), device=local)
    ens.to_device()
    tune_info = None
    if args.tune:
        from cbc_b200.autotune import Autotuner
        tuner = Autotuner(local)
        tuner.tune(ens)
        tune_info = tuner.summary()
    plan = make_plan(ens, args.schedule, args.max_steps)
    nbuckets = int(np.unique(scene.K).size)
    # pristine device copy of the initial state for the per-step reset
    pristine = {k: v.clone() for k, v in ens.dev.items()}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset():
        for k in ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters"):
            ens.dev[k].copy_(pristine[k])
        flush.fill_(1.0)  # write 256 MiB > L2 between steps

    for _ in range(args.warmup):
        reset()
        plan.launch()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx = _lib.default_context(local)
    launches0 = _lib.lib().cbc_kernel_launches(ctx.handle)
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for i in range(args.steps):
            reset()
            ev[i][0].record()
            plan.launch()
            ev[i][1].record()
        t1.record()
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    launches = _lib.lib().cbc_kernel_launches(ctx.handle) - launches0
    total_ms = t0.elapsed_time(t1)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    res = ens.to_host()
    adv = float(np.sum(res["t"] - ens.host["t"]))
    flops = flop_count(res["K"], res["steps"], res["lin_iters"], args.lin_solver)
    status = {int(k): int(v) for k, v in zip(*np.unique(res["status"], return_counts=True))}
    status_by_k = status_counts_by_k(res["K"], res["status"])

    total_ms_all, work_all = job_totals(total_ms, adv * args.steps, pg, dev)
    value = work_all / (total_ms_all * 1e-3)

    # end-to-end through the public API from host buffers (rank-local)
    e2e = None
    if args.e2e:
        # every input array of the ensemble goes up each step (state, offsets,
        # bubble / system / control parameters, coupling, times, counters)
        keys_in = tuple(k for k in ens.host if k != "K")
        keys_out = ("state", "t", "h", "event", "status", "steps", "rejected", "conv_ok", "conv_fail", "lin_iters")
        pin_in = {k: torch.from_numpy(np.ascontiguousarray(ens.host[k])).pin_memory() for k in keys_in}
        pin_out = {k: torch.empty_like(ens.dev[k], device="cpu").pin_memory() for k in keys_out}
        h2d = sum(v.numel() * v.element_size() for v in pin_in.values())
        d2h = sum(v.numel() * v.element_size() for v in pin_out.values())
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.e2e_steps):
            for k in keys_in:
                ens.dev[k].copy_(pin_in[k], non_blocking=True)
            flush.fill_(1.0)
            plan.launch()
            for k in keys_out:
                pin_out[k].copy_(ens.dev[k], non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        e2e_ms = a.elapsed_time(b)
        e2e = {"value": adv * args.e2e_steps / (e2e_ms * 1e-3) * (world if pg else 1), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps}

    # the side measurements (vec-env, direct solve, plain per-K, served,
    # large-K, plain study, CPU baseline) run in the 1-GPU job only: under
    # torchrun the other ranks would wait for them at the final barrier
    solo = world == 1
    env_lat = None
    if args.env and solo:
        env_lat = env_step_latency(local)

    lu = None
    if args.lu and solo:
        lu = lu_arm(scene, local, args.schedule, flush, args.max_steps, plain=args.plain, tune=args.tune)
        lu["alone_latency"] = alone_latency(scene, local, "lu")

    plain = None
    if args.plain and solo:
        from cbc_b200 import scenes as _sc
        n_plain = scene.ns if args.plain_ns <= 0 else min(args.plain_ns, scene.ns)
        sub = _sc.subset(scene, np.arange(n_plain))
        pv, ptime = plain_per_k(sub, dev)
        # on the whole ensemble the batched number is the timed one above (this rank's)
        bv = (adv / (float(np.max(kern_ms)) * 1e-3)) if n_plain == scene.ns else batched_once(sub, local, args.schedule)
        plain = {"value": pv, "unit": UNIT, "seconds": ptime, "systems": sub.ns, "batched_same_systems": bv,
                 "how": "reference-layout solve per K (relaunch every 2048 steps + host completion check) "
                        "on the same systems, one K after another; batched_same_systems is the batched "
                        "form on exactly those systems (the slowest timed step when they are the whole "
                        "ensemble)"}

    if rank == 0:
        peak = measured_fp64_peak(dev)
        mean_ms = float(np.mean(kern_ms))
        achieved = flops / (mean_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(args, world), "autotune": tune_info},
            "work": {"advanced_system_periods_per_step": adv, "nominal_system_periods": float(np.sum(scene.t_end)),
                     "status_counts": status, "status_counts_by_K": status_by_k,
                     "steps_per_solve": int(np.sum(res["steps"])),
                     "richardson_sweeps_per_rhs": float(np.sum(res["lin_iters"]) / max(1, 6 * np.sum(res["steps"]))),
                     "algorithmic_gflop_per_step": flops / 1e9},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": TRAFFIC_K8_BYTES,
                         "traffic_note": "DRAM bytes (read + write) of one ensemble_kernel<8,8> launch over the "
                                         "K = 8 bucket filling the GPU, ncu capture in profiles/"
                                         "ensemble_kernel_k8_richardson_steady_state.md: the state, parameters "
                                         "and coupling are read once per launch and stay on chip; traffic does "
                                         "not grow with the steps taken",
                         "note": "algorithmic FP64 flops (transcendentals counted as 1) / graph time; "
                                 "peak = cuBLAS FP64 GEMM measured in this run"},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "step_ms": [round(float(x), 1) for x in kern_ms],
        }
        hist = getattr(plan, "history", None)
        if hist:
            line["schedule_last_solve"] = [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in h.items()}
                                          for h in hist]
        if plain:
            line["plain"] = plain
            line["batched_vs_plain"] = plain["batched_same_systems"] / plain["value"]
        if e2e:
            line["e2e"] = e2e
        if env_lat:
            line["env_step_latency"] = env_lat
        if solo:
            line["alone_latency"] = alone_latency(scene, local, "richardson")
        if args.served and solo:
            line["served"] = {"offered_20k": served_measure(local, 20000.0, args.serve_seconds),
                              "below_capacity_500": served_measure(local, 500.0, args.serve_seconds)}
        if args.large_k and solo:
            line["large_k"] = large_k_measure(local, peak_tflops=peak)
        if args.plain_study and solo:
            line["plain_study"] = plain_study_measure(local)
        if lu:
            lu["roofline_frac"] = lu["achieved_tflops"] / peak
            line["lin_solver_lu"] = lu
        if solo and args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(scene)
        print(json.dumps(line), flush=True)
    plan.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def cost_tables(dev_index: int = 0, seconds: float = 0.5):
    """Per-K cost tables of the adaptive scheduler: the steady cost of one
    step attempt with the GPU full (ns: the K bucket of the mixed-K workload,
    a device-time slice of `seconds` from t = 0), the latency of one attempt
    of a system alone (us) and, from the same slice, the latency one attempt
    sees inside the full GPU (us, 90th percentile of the systems' attempt
    counts) over the alone latency (the load factor)."""
    import torch
    from cbc_b200 import scenes
    from cbc_b200.ensemble import Ensemble
    torch.cuda.set_device(dev_index)
    mix = scenes.mixed_k(ns=65536, seed=1)
    one = scenes.uniform(1, ns=26214, periods=20.0, seed=91)
    step_ns, alone_us, bulk_us = {}, {}, {}
    for k in (1, 2, 3, 4, 6, 8):
        sc = one if k == 1 else scenes.subset(mix, np.nonzero(mix.K == k)[0])
        ens = Ensemble.from_scene(sc, device=dev_index).to_device()
        ens.solve(200)
        ens.reset_device()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ens.solve(MAX_STEPS, budget_ns=int(seconds * 1e9))
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        att = (ens.dev["steps"] + ens.dev["rejected"]).cpu().numpy().astype(np.float64)
        step_ns[k] = ms * 1e6 / float(att.sum())
        bulk_us[k] = ms * 1e3 / float(np.percentile(att, 90))
        alone_us[k] = alone_latency(sc if k == 1 else mix, dev_index, "richardson", ks=(k,))[f"K{k}_us_per_attempt"]
    return {"workload": "cost_tables", "slice_s": seconds, "step_ns": step_ns, "alone_us": alone_us,
            "bulk_us": bulk_us, "load_factor": {k: bulk_us[k] / alone_us[k] for k in step_ns}}


def run_alone(args):
    """Per-attempt latency of single systems alone, both coupling solvers:
    K = 1..8 from the mixed-K workload's distributions, 16 and 32 from
    uniform scenes.  One JSON line."""
    import torch
    from cbc_b200 import scenes
    torch.cuda.set_device(0)
    mix = scenes.mixed_k(ns=args.ns, seed=1)
    extra = []
    for k in (1, 5, 7, 16, 32):
        u = scenes.uniform(k, ns=4, periods=3.0, seed=90 + k, pa_hi=1.2 if k > 8 else 1.5,
                           x_range=(-0.5, 0.5) if k > 8 else (-0.25, 0.25))
        extra.append(u)
    sc = scenes.concat(mix, *extra)
    ks = (1, 2, 3, 4, 5, 6, 7, 8, 16, 32)
    out = {"workload": "alone_latency", "unit": "us per step attempt",
           "richardson": alone_latency(sc, 0, "richardson", ks=ks), "lu": alone_latency(sc, 0, "lu", ks=ks)}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ns", type=int, default=65536)
    ap.add_argument("--no-plain", dest="plain", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-env", dest="env", action="store_false")
    ap.add_argument("--no-served", dest="served", action="store_false",
                    help="skip the served-stream measurement (Poisson 20k req/s and 500 req/s)")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--no-plain-study", dest="plain_study", action="store_false",
                    help="skip the plain parameter study (1,024 x K = 2, 10 periods) through Model.solve")
    ap.add_argument("--no-large-k", dest="large_k", action="store_false",
                    help="skip the large-K dense-output measurement")
    ap.add_argument("--workload", default="mixed_k", choices=["mixed_k", "alone", "large_k", "served", "costs"],
                    help="alone: only the single-system step latency of both coupling solvers; large_k: only "
                         "the large-K dense-output measurement (--ns systems of K = 32, --periods); served: "
                         "only the served streams (20k and 500 req/s, --serve-seconds); costs: the per-K cost "
                         "tables of the adaptive scheduler")
    ap.add_argument("--periods", type=float, default=0.5, help="span of the large_k workload")
    ap.add_argument("--lin-solver", default="richardson", choices=["richardson", "lu"],
                    help="implicit-coupling solver of the headline arm (richardson: the reference's)")
    ap.add_argument("--only-k", type=int, default=0,
                    help="keep only the systems of this K (profiling a single bucket that fills the GPU)")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the autotuner (default launch shape for every K)")
    ap.add_argument("--no-lu", dest="lu", action="store_false",
                    help="skip the direct coupling-solve (lin_solver=lu) arm on the same workload")
    ap.add_argument("--plain-ns", type=int, default=0,
                    help="systems used for the batched-vs-plain ratio (0: the whole ensemble)")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--max-steps", type=int, default=MAX_STEPS,
                    help="step cap per system (the reference's max_steps); small values make short profiling cases")
    ap.add_argument("--slices", default="",
                    help="device-time slices (s) of the adaptive schedule before its last, unbounded one, "
                         "comma separated (default 1,2,4,8)")
    ap.add_argument("--load-factor", type=float, default=0.0,
                    help="latency-lane criterion of the adaptive schedule (0: the default)")
    ap.add_argument("--schedule", default="adaptive", choices=["adaptive", "pilot", "span"],
                    help="pilot: measured longest-first re-ordering after a pilot pass; span: longest span first")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.slices:
        ADAPTIVE_OPTS["slices"] = tuple(float(x) for x in args.slices.split(","))
    if args.load_factor > 0:
        ADAPTIVE_OPTS["load_factor"] = args.load_factor
    if args.workload == "alone":
        run_alone(args)
    elif args.workload == "large_k":
        import torch
        torch.cuda.set_device(0)
        line = large_k_measure(0, ns=args.ns, periods=args.periods)
        line.update({"metric": METRIC, "n_gpus": 1, "dtype": "f64", "data": "synthetic"})
        print(json.dumps(line), flush=True)
    elif args.workload == "costs":
        print(json.dumps(cost_tables(0)), flush=True)
    elif args.workload == "served":
        import torch
        torch.cuda.set_device(0)
        line = {"workload": "served", "metric": METRIC, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
                "offered_20k": served_measure(0, 20000.0, args.serve_seconds),
                "below_capacity_500": served_measure(0, 500.0, args.serve_seconds)}
        print(json.dumps(line), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
