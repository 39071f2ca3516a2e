"""Generate golden vectors by running the REFERENCE numba integrator.

Runs kalmi901/coupled-bubble-control's own CKM1D model and its default numba
backend (``CKM1D(...).solve()`` -> ``backends/numba/rkck45_coupled_numba_solver.py``
-> ``rkck45_coupled_numba_stepper.make_kernel``) under numba's CUDA simulator
(NUMBA_ENABLE_CUDASIM=1) on the CPU of the build container, and stores the
initial host buffers together with the reference's final buffers in
``golden_ref_numba.npz``.  The reference tree (a checkout of the reference
repository) is read from the REFERENCE_ROOT environment variable, which must
be set; it is not needed anywhere else.  GOLDEN_SET=long or
GOLDEN_SET=k8 / k16 / fields / events selects the longer-span, K = 8, K = 16,
the SW_N / CONST multi-bubble or the collision-event cases.

The simulator lacks a few features the reference relies on; these shims are
applied before importing it and change no arithmetic:
  * stub modules for cupy and matplotlib (imported but unused on this path);
  * ``numba.cuda.cudadrv.devicearray.DeviceNDArray`` aliased to the
    simulator's array type; ``cuda.default_stream`` returns stream 0;
  * jit keyword arguments the simulator does not know are dropped;
  * ``cuda.shfl_sync``/``cuda.activemask`` implemented with a block barrier
    exchange.  This is exact when every thread of the block takes part, so the
    cases use one system per block and K a power of two (TILE == UPS);
  * the device helper ``sign(x) = (x > 0) - (x < 0)`` is evaluated on Python
    ints (numpy booleans cannot be subtracted in simulator mode).
Runtime is roughly a minute per case; the cases are tiny on purpose.
"""
from __future__ import annotations

import os
import sys
import threading
import types

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"

import numpy as np  # noqa: E402

REF = os.environ.get("REFERENCE_ROOT", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def install_shims():
    for name in ("cupy", "matplotlib", "matplotlib.pyplot"):
        m = types.ModuleType(name)
        m.ndarray = type("ndarray", (), {})
        sys.modules[name] = m
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    from numba import cuda
    from numba.cuda.simulator.cudadrv import devicearray as simda
    da = types.ModuleType("numba.cuda.cudadrv.devicearray")
    da.DeviceNDArray = simda.FakeCUDAArray
    sys.modules["numba.cuda.cudadrv.devicearray"] = da
    cuda.default_stream = lambda: 0

    import numba.cuda.simulator.api as simapi
    import numba.cuda.simulator.kernelapi as ka
    orig_jit = simapi.jit

    def jit(func_or_sig=None, **kw):
        keep = {k: v for k, v in kw.items() if k in ("device", "debug", "argtypes", "inline", "restype",
                                                       "fastmath", "link", "opt", "cache")}

        def wrap(fn):
            if getattr(fn, "__name__", "") == "sign":
                def sign(x):
                    return int(x > 0) - int(x < 0)
                fn = sign
            return orig_jit(**keep)(fn) if keep else orig_jit(fn)
        if callable(func_or_sig):
            return wrap(func_or_sig)
        return wrap

    cuda.jit = jit
    simapi.jit = jit

    def activemask(self):
        return 0xFFFFFFFF

    def shfl_sync(self, mask, val, src):
        th = threading.current_thread()
        mgr = th._manager
        box = mgr.__dict__.setdefault("_shfl_box", {})
        box[th.thread_id] = val
        th.syncthreads()
        out = box.get(int(src), val)
        th.syncthreads()
        return out

    ka.FakeCUDAModule.activemask = activemask
    ka.FakeCUDAModule.shfl_sync = shfl_sync


# Small cases: (name, K, ac, nk, R0 um (K), PA bar (nk), FR kHz (nk), PS (units of pi), X0, t_end)
CASES = [
    ("k2_swa", 2, "SW_A", 2, [5.0, 3.0], [1.2, 0.4], [25.0, 50.0], [0.3, 1.1], [-0.05, 0.05], 0.004),
    ("k2_swn", 2, "SW_N", 2, [6.0, 5.0], [0.5, 0.3], [25.0, 50.0], [0.0, 0.0], [-0.05, 0.05], 0.004),
    ("k2_const", 2, "CONST", 1, [7.0, 5.0], [-1.2156], [20.0], [0.0], [0.0, 200e-6 / (1497.0 / 20e3)], 0.004),
    ("k4_swa", 4, "SW_A", 2, [4.0, 6.0, 3.0, 5.0], [0.9, 0.7], [25.0, 50.0], [1.5, 0.2],
     [-0.2, -0.1, 0.05, 0.2], 0.002),
    ("k1_swa", 1, "SW_A", 2, [5.5], [1.4, 0.6], [25.0, 50.0], [0.1, 0.9], [0.1], 0.004),
]


# Longer spans (a few hundred to a thousand steps, through a collapse for the
# driven cases).  Written to golden_ref_numba_long.npz with GOLDEN_SET=long.
CASES_LONG = [
    ("k2_swa_long", 2, "SW_A", 2, [6.0, 4.0], [1.3, 0.8], [25.0, 50.0], [0.7, 1.6], [-0.1, 0.02], 0.06),
    ("k4_swa_long", 4, "SW_A", 2, [5.0, 3.5, 6.0, 4.0], [1.2, 0.7], [25.0, 50.0], [0.5, 1.4],
     [-0.2, -0.08, 0.06, 0.18], 0.03),
    ("k2_const_long", 2, "CONST", 1, [7.0, 5.0], [-1.2156], [20.0], [0.0], [0.0, 200e-6 / (1497.0 / 20e3)], 0.06),
]


# K = 8 (every partner-sum chain of the kernels holds two partners).  Written to
# golden_ref_numba_k8.npz with GOLDEN_SET=k8.
CASES_K8 = [
    ("k8_swa", 8, "SW_A", 2, [5.0, 3.0, 4.0, 6.0, 2.5, 5.5, 3.5, 4.5], [1.1, 0.6], [25.0, 50.0], [0.4, 1.3],
     [-0.35, -0.25, -0.15, -0.05, 0.05, 0.15, 0.25, 0.35], 0.001),
]


# K = 16 (the generic-K kernel: chains of three and four partners).  Written to
# golden_ref_numba_k16.npz with GOLDEN_SET=k16.
CASES_K16 = [
    ("k16_swa", 16, "SW_A", 2, [4.0 + 0.25 * (i % 7) for i in range(16)], [1.0, 0.5], [25.0, 50.0], [0.2, 0.9],
     [-0.375 + 0.05 * i for i in range(16)], 0.0005),
]


# SW_N and CONST fields with several coupled bubbles.  Written to
# golden_ref_numba_fields.npz with GOLDEN_SET=fields.
CASES_FIELDS = [
    ("k4_swn", 4, "SW_N", 2, [5.0, 4.0, 6.0, 3.0], [0.6, 0.4], [25.0, 50.0], [0.0, 0.0],
     [-0.15, -0.05, 0.05, 0.15], 0.002),
    ("k8_const", 8, "CONST", 1, [7.0, 5.0, 6.0, 4.0, 5.5, 6.5, 4.5, 5.0], [-1.0], [20.0], [0.0],
     [-0.35, -0.25, -0.15, -0.05, 0.05, 0.15, 0.25, 0.35], 0.001),
]


# Two bubbles that start just outside the collision threshold and grow into
# it: event bracketing by step rejection and the terminal status 2.  Written
# to golden_ref_numba_events.npz with GOLDEN_SET=events.
CASES_EVENTS = [
    ("k2_event", 2, "SW_A", 2, [20.0, 20.0], [1.2, 0.1], [25.0, 50.0], [0.75, 0.0], [0.0, 7.548029e-04], 0.1),
]


# Dense output (an 11th field: the number of stored points).  The reference
# keeps writing the current state into the last stored slot until the next
# slot is due (its slot flag is never reset), so its dense_state[i] holds the
# last state before sample i+1 was taken, and the last slot the final state;
# tests/test_oracle_golden.py replays that rule in the oracle's test-only
# emulation mode.  Written to golden_ref_numba_dense.npz with GOLDEN_SET=dense.
CASES_DENSE = [
    ("k2_swa_dense", 2, "SW_A", 2, [5.0, 3.0], [1.2, 0.4], [25.0, 50.0], [0.3, 1.1], [-0.05, 0.05], 0.004, 5),
    ("k4_swa_dense", 4, "SW_A", 2, [4.0, 6.0, 3.0, 5.0], [0.9, 0.7], [25.0, 50.0], [1.5, 0.2],
     [-0.2, -0.1, 0.05, 0.2], 0.002, 4),
]


# A longer span that runs through a bubble collapse (R: 1 -> 3.65 -> 0.18 ->
# 2.3, about 1,650 steps) with dense output.  Written to
# golden_ref_numba_collapse.npz with GOLDEN_SET=collapse (a few hours under the
# simulator).
CASES_COLLAPSE = [
    ("k2_collapse", 2, "SW_A", 2, [8.0, 7.5], [1.2, 0.2], [25.0, 50.0], [0.25, 0.0], [-0.1, 0.02], 0.9, 10),
]


def run_case(case, water):
    from coupledbubble_control.models import CKM1D, MaterialProperties
    from coupledbubble_control.backends import BackendName, KernelVariant
    name, K, ac, nk, R0, PA, FR, PS, X0, t_end = case[:10]
    ndo = case[10] if len(case) > 10 else 0
    ns = 1
    mp = MaterialProperties()
    if water:
        for k, v in dict(RHO=998.0, CL=1497.0, ST=0.0728, VIS=1e-3, P0=1.0e5, PV=2330.0, PE=1.4).items():
            setattr(mp, k, v)
    model = CKM1D(num_systems=ns, systems_per_block=1, units_per_system=K,
                  R0=np.array([R0], dtype=np.float64), PA=np.array(PA, dtype=np.float64)[:, None],
                  FR=np.array(FR, dtype=np.float64)[:, None], PS=np.array(PS, dtype=np.float64)[:, None],
                  REF_FREQ=FR[0], num_components=nk, acoustic_field=ac, mat_props=mp,
                  backend=BackendName.NUMBA, variant=KernelVariant.SHARED, num_stored_points=ndo)
    hb = model.runtime.host_buffers
    hb.state.time_end[:] = t_end
    hb.state.actual_state[1, :, :K] = np.array(X0)
    init = {}
    for grp in (hb.state, hb.params, hb.dense, hb.status):
        for k in grp.__dataclass_fields__:
            init[k] = np.array(getattr(grp, k), copy=True)
    model.solve(max_steps=1_000_000, kernel_steps=1_000_000, sync_to_host=True)
    final = {}
    db = model.runtime.device_buffers
    for grp_name in ("state", "status") + (("dense",) if ndo > 0 else ()):
        grp = getattr(db, grp_name)
        for k in grp.__dataclass_fields__:
            final[k] = np.array(grp.__getattribute__(k).copy_to_host(), copy=True)
    return init, final, dict(name=name, K=K, ac=ac, nk=nk, ndo=ndo)


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set REFERENCE_ROOT to a checkout of the reference repository")
    install_shims()
    sys.path.insert(0, REF)
    out = {}
    which = os.environ.get("GOLDEN_SET", "")
    sets = {"long": CASES_LONG, "k8": CASES_K8, "k16": CASES_K16, "fields": CASES_FIELDS,
            "events": CASES_EVENTS, "dense": CASES_DENSE, "collapse": CASES_COLLAPSE}
    cases = sets.get(which, CASES)
    for case in cases:
        print("running", case[0], flush=True)
        init, final, meta = run_case(case, water=True)
        for k, v in init.items():
            out[f"{meta['name']}/init/{k}"] = v
        for k, v in final.items():
            out[f"{meta['name']}/final/{k}"] = v
        out[f"{meta['name']}/meta"] = np.array([meta["K"], meta["nk"], ["CONST", "SW_N", "SW_A"].index(meta["ac"])])
        out[f"{meta['name']}/ndo"] = np.array([meta["ndo"]])
        print("  t", final["actual_time"], "R", final["actual_state"][0, 0, :meta["K"]], flush=True)
    fn = os.path.join(HERE, f"golden_ref_numba_{which}.npz" if which in sets else "golden_ref_numba.npz")
    np.savez_compressed(fn, **out)
    print("wrote", fn)


if __name__ == "__main__":
    main()
