"""Shared helpers of the parity tests: run a model through the C ABI on the
GPU and through the CPU oracle on identical host buffers, then compare."""
from __future__ import annotations

import copy

import numpy as np

from cbc_b200 import scenes
from cbc_b200.models import SolverSpec
from oracle import oracle

COMPARED = ["actual_time", "time_step", "actual_state", "actual_event", "status_flags", "dense_index",
            "dense_time", "dense_state", "total_steps", "rejected_steps", "convergece_success",
            "convergence_failures"]


def run_pair(scene, solver_spec=None, max_steps=200_000, kernel_steps=2048, launch_mode="relaunch",
             nthreads=0):
    """(gpu_buffers, oracle_buffers) as dicts of numpy arrays."""
    import torch
    from cbc_b200.backends import b200_solver

    model = scenes.build_model(scene, solver_spec=solver_spec)
    host = copy.deepcopy(oracle.model_buffers(model))
    # GPU through the model API (Model.solve -> backend solver -> C ABI)
    model._ensure_buffers()
    lin = torch.zeros(model._execution_spec.ns, dtype=torch.int64, device="cuda")
    kern = b200_solver.load_kernel(model._model_spec, model._execution_spec, model._solver_spec, launch_mode)
    b200_solver.solver(kern, model.runtime.device_buffers, model._model_spec, model._execution_spec,
                       model._solver_spec, max_steps=max_steps, kernel_steps=kernel_steps, lin_iters=lin)
    torch.cuda.synchronize()
    db = model.runtime.device_buffers
    gpu = {}
    for grp in (db.state, db.params, db.dense, db.status):
        for k in grp.__slots__:
            gpu[k] = getattr(grp, k).cpu().numpy()
    gpu["lin_iters"] = lin.cpu().numpy()
    # oracle on a copy of the initial host buffers
    es, ms = model._execution_spec, model._model_spec
    spec = oracle.make_spec(es.ns, es.ups, es.tile, es.ndo, ms.nk, ms.ac, model._solver_spec)
    launches = (max_steps + kernel_steps - 1) // kernel_steps
    oracle.solve_ref_layout(spec, host, launches * kernel_steps, nthreads)
    return gpu, host


def assert_bit_exact(gpu, ref, keys=COMPARED):
    for k in keys + ["lin_iters"]:
        a, b = gpu[k], ref[k]
        if a.size == 0:
            continue
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        if not np.all(same):
            bad = np.argwhere(~same)
            i = tuple(bad[0])
            raise AssertionError(f"{k}: {len(bad)} mismatches, first at {i}: gpu={a[i]!r} oracle={b[i]!r}")


def max_rel_err(a, b, floor):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def ensemble_uniform_to_ref(h, K, nk):
    """Reference-layout host buffers (tile = K) from the ragged arrays of a
    uniform-K ensemble, for running the oracle on ensemble state."""
    ns = h["t"].shape[0]
    st = h["state"].reshape(ns, K, 4)
    up = h["unit_params"].reshape(ns, K, -1)[:, :, :13]
    cm = h["coupling"].reshape(ns, 3, K, K)
    return {
        "actual_time": h["t"].copy(), "time_end": h["t_end"].copy(), "time_begin": h["t_begin"].copy(),
        "time_step": h["h"].copy(), "actual_state": np.ascontiguousarray(np.transpose(st, (2, 0, 1))),
        "unit_params": np.ascontiguousarray(np.transpose(up, (2, 0, 1))),
        "system_params": np.ascontiguousarray(h["system_params"][:, :5].T),
        "control_params": np.ascontiguousarray(h["control_params"][:, :4 * nk].T),
        "coupling_matrices": np.ascontiguousarray(np.transpose(cm, (1, 2, 0, 3))),
        "dense_index": np.zeros(ns, np.int32), "dense_time": np.zeros((0, ns)),
        "dense_state": np.zeros((0, 4, ns, K)), "actual_event": h["event"].copy(),
        "status_flags": h["status"].copy(), "total_steps": np.zeros(ns, np.int32),
        "rejected_steps": np.zeros(ns, np.int32), "convergece_success": np.zeros(ns, np.int32),
        "convergence_failures": np.zeros(ns, np.int32), "lin_iters": np.zeros(ns, np.int64),
    }
