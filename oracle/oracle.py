"""ctypes front end of the CPU oracle (test infrastructure only).

Used by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline leg to
check or time the CUDA library.  Never imported by the product package.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_AC = {"CONST": 0, "SW_N": 1, "SW_A": 2}
# "reference_defect" (oracle only): the reference's dense output as it is,
# with its slot overwrite, for pinning against the reference's own samples
_DENSE = {"reference": 0, "grid": 1, "reference_defect": 2}
_LIN = {"richardson": 0, "lu": 1}


class cbo_spec(ctypes.Structure):
    _fields_ = [("ns", ctypes.c_int32), ("ups", ctypes.c_int32), ("tile", ctypes.c_int32),
                ("ndo", ctypes.c_int32), ("nk", ctypes.c_int32), ("ac", ctypes.c_int32),
                ("dense_mode", ctypes.c_int32), ("lin_max_iter", ctypes.c_int32),
                ("atol", ctypes.c_double), ("rtol", ctypes.c_double), ("min_step", ctypes.c_double),
                ("max_step", ctypes.c_double), ("lin_atol", ctypes.c_double),
                ("lin_rtol", ctypes.c_double), ("lin_relaxation", ctypes.c_double),
                ("etol", ctypes.c_double), ("col_threshold", ctypes.c_double),
                ("lin_solver", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def _cpu_has_fma() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " fma " in line + " "
    except OSError:
        pass
    return False


_lib = None


def lib():
    """Load the oracle library, building it with make if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    name = "libckm1d_oracle_fma.so" if _cpu_has_fma() else "libckm1d_oracle.so"
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        import subprocess
        subprocess.check_call(["make", "-s", "-C", _HERE])
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    L.cbo_solve_ref_layout.argtypes = [ctypes.POINTER(cbo_spec)] + [P] * 19 + [ctypes.c_int64, ctypes.c_int32]
    L.cbo_solve_ref_layout.restype = ctypes.c_int
    L.cbo_math_eval.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P]
    L.cbo_math_eval.restype = None
    L.cbo_lu_solve.argtypes = [ctypes.c_int32, P, P]
    L.cbo_lu_solve.restype = ctypes.c_int
    _lib = L
    return L


def make_spec(ns, ups, tile, ndo, nk, ac, solver_spec) -> cbo_spec:
    s = solver_spec
    return cbo_spec(ns, ups, tile, ndo, nk, _AC[ac] if isinstance(ac, str) else int(ac),
                    _DENSE[getattr(s, "dense_mode", "reference")], int(s.lin_max_iter), s.atol, s.rtol,
                    s.min_step, s.max_step, s.lin_atol, s.lin_rtol, s.lin_relaxation, s.etol,
                    getattr(s, "col_threshold", 0.1), _LIN[getattr(s, "lin_solver", "richardson")], 0)


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle buffers must be C-contiguous"
    return a.ctypes.data


def solve_ref_layout(spec: cbo_spec, b: Dict[str, np.ndarray], budget: int, nthreads: int = 0) -> None:
    """Integrate in place on host numpy buffers of the reference layout.

    ``b`` keys: actual_time, time_end, time_begin, time_step, actual_state,
    unit_params, system_params, control_params, coupling_matrices,
    dense_index, dense_time, dense_state, actual_event, status_flags and the
    optional counters total_steps, rejected_steps, convergece_success,
    convergence_failures, lin_iters.
    """
    keys = ["actual_time", "time_end", "time_begin", "time_step", "actual_state", "unit_params",
            "system_params", "control_params", "coupling_matrices", "dense_index", "dense_time",
            "dense_state", "actual_event", "status_flags", "total_steps", "rejected_steps",
            "convergece_success", "convergence_failures", "lin_iters"]
    ptrs = [_p(b.get(k)) for k in keys]
    rc = lib().cbo_solve_ref_layout(ctypes.byref(spec), *ptrs, int(budget), int(nthreads))
    if rc != 0:
        raise ValueError(f"oracle rejected the arguments (code {rc})")


def model_buffers(model) -> Dict[str, np.ndarray]:
    """Flat dict view of a CKM1D model's host buffers (plus a lin_iters counter)."""
    hb = model.runtime.host_buffers
    d = {}
    for grp in (hb.state, hb.params, hb.dense, hb.status):
        for k in grp.__slots__:
            d[k] = getattr(grp, k)
    d["lin_iters"] = np.zeros(model._execution_spec.ns, dtype=np.int64)
    return d


def solve_model(model, max_steps: int = 100_000, kernel_steps: int = 2048, nthreads: int = 0):
    """Oracle counterpart of ``model.solve()`` on the model's host buffers.

    The step budget per system equals what the reference's relaunch loop
    allows: ceil(max_steps / kernel_steps) launches of kernel_steps steps.
    """
    es, ms = model._execution_spec, model._model_spec
    spec = make_spec(es.ns, es.ups, es.tile, es.ndo, ms.nk, ms.ac, model._solver_spec)
    buf = model_buffers(model)
    launches = (max_steps + kernel_steps - 1) // kernel_steps
    solve_ref_layout(spec, buf, launches * kernel_steps, nthreads)
    return buf


def math_eval(kind: int, x: np.ndarray, y: Optional[np.ndarray] = None) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    yy = np.ascontiguousarray(y if y is not None else np.zeros_like(x), dtype=np.float64)
    out = np.empty_like(x)
    lib().cbo_math_eval(kind, x.size, x.ctypes.data, yy.ctypes.data, out.ctypes.data)
    return out


def lu_solve(a: np.ndarray):
    """The oracle's direct coupling solve on one augmented 2K x (2K+1) matrix:
    (x, ok, eliminated matrix)."""
    a = np.array(a, dtype=np.float64, order="C", copy=True)
    n = a.shape[0]
    assert n % 2 == 0 and a.shape == (n, n + 1)
    x = np.zeros(n)
    rc = lib().cbo_lu_solve(n // 2, a.ctypes.data, x.ctypes.data)
    if rc < 0:
        raise ValueError("bad K")
    return x, bool(rc), a
