"""ctypes binding of libcbc_b200.so (the C ABI in include/cbc_b200.h).

The library is built in-tree by ``csrc/Makefile`` (``python -m cbc_b200.build``
or ``__graft_entry__.build()``).  There is no fallback: if the shared object is
missing, :func:`lib` raises, and a solve never runs anywhere but on the GPU.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcbc_b200.so")

P = ctypes.c_void_p
i32 = ctypes.c_int32
i64 = ctypes.c_int64
f64 = ctypes.c_double

# status codes (include/cbc_b200.h; reference rkck45_coupled_numba_stepper.py:27-33)
ACTIVE, SUCCESS, EVENT_TERMINAL = 0, 1, 2
MAX_STEPS_REACHED, STEP_SIZE_LIMIT, CONVERGENCE_FAILURE, SINGULARITY_OR_NAN = -1, -2, -3, -4
LAUNCH_RELAUNCH, LAUNCH_SINGLE = 0, 1
AC_CODES = {"CONST": 0, "SW_N": 1, "SW_A": 2}
DENSE_CODES = {"reference": 0, "grid": 1}
LIN_CODES = {"richardson": 0, "lu": 1}


class cbc_spec(ctypes.Structure):
    _fields_ = [("ns", i32), ("ups", i32), ("tile", i32), ("ndo", i32), ("nk", i32), ("ac", i32),
                ("dense_mode", i32), ("lin_max_iter", i32), ("atol", f64), ("rtol", f64),
                ("min_step", f64), ("max_step", f64), ("lin_atol", f64), ("lin_rtol", f64),
                ("lin_relaxation", f64), ("etol", f64), ("col_threshold", f64), ("lin_solver", i32),
                ("reserved", i32)]


class cbc_buffers(ctypes.Structure):
    _fields_ = [(n, P) for n in (
        "actual_time", "time_end", "time_begin", "time_step", "actual_state", "unit_params",
        "system_params", "control_params", "coupling_matrices", "dense_index", "dense_time",
        "dense_state", "actual_event", "status_flags", "total_steps", "rejected_steps",
        "convergence_success", "convergence_failures", "lin_iters")]


class cbc_solve_stats(ctypes.Structure):
    _fields_ = [("launches", i32), ("active_left", i32), ("device_ms", f64)]


class cbc_ensemble(ctypes.Structure):
    _fields_ = [("ns", i32), ("up_stride", i32), ("sp_stride", i32), ("cp_stride", i32), ("nb", i64)] + \
        [(n, P) for n in ("bubble_offset", "coupling_offset", "state", "unit_params", "system_params",
                          "control_params", "coupling", "t", "t_end", "t_begin", "h", "event", "status",
                          "dense_index", "dense_time", "dense_state", "steps", "rejected", "conv_ok",
                          "conv_fail", "lin_iters", "trace_load_ns", "trace_done_ns")]


class cbc_work(ctypes.Structure):
    _fields_ = [("order", P), ("nbuckets", i32), ("bucket_K", P), ("bucket_begin", P), ("threads", P),
                ("blocks_per_sm", P), ("share", P), ("exclusive", P), ("budget_ns", i64),
                ("steps_total", i32), ("reserved", i32), ("slots", P), ("min_blocks", P)]


class cbc_env_io(ctypes.Structure):
    _fields_ = [("actions", P), ("n_act", i32), ("act_stride", i32), ("act_scale", f64), ("obs", P),
                ("failed", P), ("K", i32), ("pad", i32), ("t_span", f64), ("h0", f64)] + \
        [(n, P) for n in ("targets", "rewards", "terminated", "time_outs", "done", "algo_steps", "total_rewards",
                          "final_obs", "episode_return", "episode_len", "reset_count")] + \
        [(n, f64) for n in ("position_tolerance", "r_dnorm", "reward_exp", "w_dist", "w_intensity", "pos_reward",
                            "neg_reward", "min_distance", "max_distance", "domain_lo", "domain_hi")] + \
        [("episode_length", i32), ("pad2", i32), ("seed", ctypes.c_uint64)]


class cbc_precompute_consts(ctypes.Structure):
    _fields_ = [(n, f64) for n in ("two_pi", "pi", "w_ref", "l_ref", "rho", "cl", "p0", "pv", "st2", "k1", "p0pv",
                                   "k4", "tw", "k6", "hl", "k9", "k10", "k11", "km2")] + \
        [("system_params", f64 * 5)]


def admit_record_len(nk: int) -> int:
    """Doubles per request record of cbc_admit (CBC_ADMIT_RECORD)."""
    return 5 + 3 * int(nk) + 64


class CBCError(RuntimeError):
    """A C-ABI call returned a negative code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"cbc error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C coupled-bubble-control_b200/csrc` "
                "(the CKM1D solver has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.cbc_version.restype = i32
        L.cbc_version.argtypes = []
        L.cbc_create.restype = i32
        L.cbc_create.argtypes = [ctypes.POINTER(P), i32]
        L.cbc_destroy.restype = i32
        L.cbc_destroy.argtypes = [P]
        L.cbc_last_error.restype = ctypes.c_char_p
        L.cbc_last_error.argtypes = [P]
        L.cbc_solve.restype = i32
        L.cbc_solve.argtypes = [P, ctypes.POINTER(cbc_spec), ctypes.POINTER(cbc_buffers), i64, i32, i32, P,
                                ctypes.POINTER(cbc_solve_stats)]
        _declare_extra(L)
        _lib = L
        return L


def _declare_extra(L) -> None:
    """Signatures of the entry points added after the reference-layout solver."""
    for name, res, args in EXTRA_SIGNATURES:
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args


EXTRA_SIGNATURES: list = [
    ("cbc_ensemble_solve", i32, [P, ctypes.POINTER(cbc_spec), ctypes.POINTER(cbc_ensemble),
                                 ctypes.POINTER(cbc_work), i64, P]),
    ("cbc_plan_create", i32, [P, ctypes.POINTER(cbc_spec), ctypes.POINTER(cbc_ensemble),
                              ctypes.POINTER(cbc_work), i64, ctypes.POINTER(P)]),
    ("cbc_env_plan_create", i32, [P, ctypes.POINTER(cbc_spec), ctypes.POINTER(cbc_ensemble),
                                  ctypes.POINTER(cbc_work), i64, ctypes.POINTER(cbc_env_io), ctypes.POINTER(P)]),
    ("cbc_ensemble_solve_noalloc", i32, [P, ctypes.POINTER(cbc_spec), ctypes.POINTER(cbc_ensemble),
                                         ctypes.POINTER(cbc_work), i64, P]),
    ("cbc_admit", i32, [P, ctypes.POINTER(cbc_ensemble), ctypes.POINTER(cbc_precompute_consts), P, i32, i32, i64,
                        P]),
    ("cbc_env_reset", i32, [P, ctypes.POINTER(cbc_ensemble), ctypes.POINTER(cbc_env_io), P, P]),
    ("cbc_plan_launch", i32, [P, P]),
    ("cbc_kernel_launches", i64, [P]),
    ("cbc_plan_destroy", i32, [P]),
]


def check(rc: int, ctx: Optional[int] = None) -> None:
    if rc != 0:
        msg = lib().cbc_last_error(ctx).decode("utf-8", "replace")
        raise CBCError(rc, msg)


class Context:
    """Owns one ``cbc_context`` on a CUDA device."""

    def __init__(self, device: int = 0):
        h = P()
        check(lib().cbc_create(ctypes.byref(h), int(device)))
        self.handle = h.value
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().cbc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> None:
        check(rc, self.handle)


_contexts = {}


def default_context(device: Optional[int] = None) -> Context:
    """Process-wide context per device (created on first use)."""
    if device is None:
        import torch
        device = torch.cuda.current_device()
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[device] = ctx
    return ctx
