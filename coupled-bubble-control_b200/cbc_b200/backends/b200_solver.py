"""B200 backend solver: the drop-in for the reference's backend ``solver``.

Same call signature and return value as
``coupledbubble_control/backends/numba/rkck45_coupled_numba_solver.py:8-18``
and ``backends/cupy_cuda/rkck45_coupled_cupy_solver.py:8-18``:
``solver(kernel, d_buffers, model_spec, execution_spec, solver_spec, max_steps,
kernel_steps=2048, benchmark=False, debug=False)`` -> list of per-launch times
(seconds) when ``benchmark`` else ``None``.  ``d_buffers`` is the model's
device ``BufferSet`` (torch CUDA tensors); the library updates it in place
through raw pointers.

``kernel`` is the handle returned by :func:`load_kernel`.  Launch behaviour:
``launch_mode="relaunch"`` (default) keeps the reference's host loop (one
launch per ``kernel_steps`` followed by a completion check);
``"single"`` spends the whole budget in one launch without host round trips.
Results are identical in both modes.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional

from .. import _lib
from ..models.buffers import data_ptr


@dataclass
class KernelHandle:
    spec: _lib.cbc_spec
    launch_mode: str = "relaunch"
    device: Optional[int] = None


def make_cbc_spec(model_spec, execution_spec, solver_spec) -> _lib.cbc_spec:
    s = solver_spec
    return _lib.cbc_spec(
        int(execution_spec.ns), int(execution_spec.ups), int(execution_spec.tile), int(execution_spec.ndo),
        int(model_spec.nk), _lib.AC_CODES[model_spec.ac], _lib.DENSE_CODES[getattr(s, "dense_mode", "reference")],
        int(s.lin_max_iter), float(s.atol), float(s.rtol), float(s.min_step), float(s.max_step),
        float(s.lin_atol), float(s.lin_rtol), float(s.lin_relaxation), float(s.etol),
        float(getattr(s, "col_threshold", 0.1)), _lib.LIN_CODES[getattr(s, "lin_solver", "richardson")], 0)


def load_kernel(model_spec, execution_spec, solver_spec, launch_mode: str = "relaunch") -> KernelHandle:
    """Counterpart of the reference's kernel build step (``make_kernel`` /
    ``load_coupled_kernel``).  Nothing is compiled at run time: the sm_100a
    library is prebuilt; this validates that it loads and packs the spec."""
    _lib.lib()
    return KernelHandle(make_cbc_spec(model_spec, execution_spec, solver_spec), launch_mode)


def _check_tensor(name, t, dtype_name: str, shape):
    import torch
    if t is None:
        return
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA torch tensor")
    if str(t.dtype) != dtype_name:
        raise TypeError(f"{name} must be {dtype_name}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} shape mismatch: expected {tuple(shape)}, got {tuple(t.shape)}")


def pack_buffers(d_buffers, spec: _lib.cbc_spec, lin_iters=None) -> _lib.cbc_buffers:
    ns, tile, ups, ndo, nk = spec.ns, spec.tile, spec.ups, spec.ndo, spec.nk
    st, pr, de, su = d_buffers.state, d_buffers.params, d_buffers.dense, d_buffers.status
    f64, i32 = "torch.float64", "torch.int32"
    for name, t, dt, shp in (
            ("actual_time", st.actual_time, f64, (ns,)), ("time_end", st.time_end, f64, (ns,)),
            ("time_begin", st.time_begin, f64, (ns,)), ("time_step", st.time_step, f64, (ns,)),
            ("actual_state", st.actual_state, f64, (4, ns, tile)),
            ("unit_params", pr.unit_params, f64, (13, ns, tile)),
            ("system_params", pr.system_params, f64, (5, ns)),
            ("control_params", pr.control_params, f64, (4 * nk, ns)),
            ("coupling_matrices", pr.coupling_matrices, f64, (3, ups, ns, tile)),
            ("actual_event", su.actual_event, f64, (ns,)), ("status_flags", su.status_flags, i32, (ns,))):
        _check_tensor(name, t, dt, shp)
    if ndo > 0:
        _check_tensor("dense_index", de.dense_index, i32, (ns,))
        _check_tensor("dense_time", de.dense_time, f64, (ndo, ns))
        _check_tensor("dense_state", de.dense_state, f64, (ndo, 4, ns, tile))
    b = _lib.cbc_buffers()
    b.actual_time = data_ptr(st.actual_time)
    b.time_end = data_ptr(st.time_end)
    b.time_begin = data_ptr(st.time_begin)
    b.time_step = data_ptr(st.time_step)
    b.actual_state = data_ptr(st.actual_state)
    b.unit_params = data_ptr(pr.unit_params)
    b.system_params = data_ptr(pr.system_params)
    b.control_params = data_ptr(pr.control_params)
    b.coupling_matrices = data_ptr(pr.coupling_matrices)
    if ndo > 0:
        b.dense_index = data_ptr(de.dense_index)
        b.dense_time = data_ptr(de.dense_time)
        b.dense_state = data_ptr(de.dense_state)
    b.actual_event = data_ptr(su.actual_event)
    b.status_flags = data_ptr(su.status_flags)
    for fld, t in (("total_steps", su.total_steps), ("rejected_steps", su.rejected_steps),
                   ("convergence_success", su.convergece_success),
                   ("convergence_failures", su.convergence_failures)):
        if t is not None:
            _check_tensor(fld, t, i32, (ns,))
            setattr(b, fld, data_ptr(t))
    if lin_iters is not None:
        _check_tensor("lin_iters", lin_iters, "torch.int64", (ns,))
        b.lin_iters = data_ptr(lin_iters)
    return b


def solver(kernel: KernelHandle, d_buffers, model_spec, execution_spec, solver_spec, max_steps: int,
           kernel_steps: int = 2048, benchmark: bool = False, debug: bool = False,
           lin_iters=None, stream=None) -> Optional[List[float]]:
    import torch
    spec = kernel.spec
    b = pack_buffers(d_buffers, spec, lin_iters)
    dev = d_buffers.state.actual_state.device.index
    ctx = _lib.default_context(dev)
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    stats = _lib.cbc_solve_stats()
    mode = _lib.LAUNCH_SINGLE if kernel.launch_mode == "single" else _lib.LAUNCH_RELAUNCH
    with torch.cuda.device(dev):
        ctx.check(_lib.lib().cbc_solve(ctx.handle, ctypes.byref(spec), ctypes.byref(b), int(max_steps),
                                       int(kernel_steps), mode, ctypes.c_void_p(stream.cuda_stream),
                                       ctypes.byref(stats) if (benchmark or debug) else None))
    if debug:
        print(f"B200 CKM1D solver: launches={stats.launches} active_left={stats.active_left} "
              f"device_ms={stats.device_ms:.3f}")
    if benchmark:
        n = max(int(stats.launches), 1)
        return [stats.device_ms * 1e-3 / n] * n
    return None
