"""Model base class: buffers, shape checks and ``solve()``.

Mirrors ``coupledbubble_control/models/model.py``: ``MaterialProperties``
(:16-24), ``ModelRuntime`` (:27-41), ``Model`` with the shape properties
(:56-106), ``solve`` (:108-162), host-buffer initialisation (:180-225),
``_ensure_buffers`` (:227-238) and the shape checks (:241-279).  ``solve``
keeps the reference signature and return value (list of launch times when
``benchmark`` is set, else ``None``).
"""
from __future__ import annotations

from typing import Any, Callable, Dict, Optional, Tuple

import numpy as np

from .buffers import (ActualStateBuffer, BufferOps, BufferSet, DenseOutputBuffer,
                      ParameterBuffer, StatusBuffer)
from .specs import ExecutionSpec, LayoutEntry, ModelSpec, SolverSpec
from ..backends import BackendName, KernelVariant


class MaterialProperties:
    """Liquid properties in SI units.  Defaults are the reference's
    (models/model.py:16-24); pass keyword arguments to override."""

    PV = 0.0          # vapour pressure [Pa]
    RHO = 998.0       # density [kg/m^3]
    ST = 0.0725       # surface tension [N/m]
    VIS = 0.001       # viscosity [Pa s]
    CL = 1500         # sound speed [m/s]
    P0 = 1.013 * 1e5  # ambient pressure [Pa]
    PE = 1.4          # polytropic exponent [-]

    def __init__(self, **overrides: float) -> None:
        for k, v in overrides.items():
            if not hasattr(type(self), k):
                raise AttributeError(f"unknown material property {k!r}")
            setattr(self, k, float(v))


def water() -> MaterialProperties:
    """Water at room temperature as used by the parameter-study workloads:
    rho 998 kg/m^3, c 1497 m/s, sigma 0.0728 N/m, mu 1e-3 Pa s,
    P_inf 1 bar, p_vap 2.33 kPa, polytropic exponent 1.4."""
    return MaterialProperties(RHO=998.0, CL=1497.0, ST=0.0728, VIS=1e-3, P0=1.0e5, PV=2330.0, PE=1.4)


class ModelRuntime:
    def __init__(self, backend: BackendName, variant: KernelVariant, stream=None) -> None:
        self.backend = backend
        self.variant = variant
        self.stream = stream
        self.host_buffers: BufferSet
        self.device_buffers: Optional[BufferSet] = None
        self.solver: Optional[Callable] = None


class Model:
    _model_spec: ModelSpec
    _execution_spec: ExecutionSpec
    _solver_spec: SolverSpec
    _available_backends: Tuple[BackendName, ...]
    runtime: ModelRuntime
    buffer_ops: BufferOps
    control_layout: Dict[str, LayoutEntry]
    state_layout: Dict[str, LayoutEntry]

    # ---- shapes (reference model.py:56-106) ----
    @property
    def time_shape(self):
        return (self._execution_spec.ns,)

    @property
    def state_shape(self):
        return (self._model_spec.sd, self._execution_spec.ns, self._execution_spec.tile)

    @property
    def unit_param_shape(self):
        return (self._model_spec.nup, self._execution_spec.ns, self._execution_spec.tile)

    @property
    def system_param_shape(self):
        return (self._model_spec.nsp, self._execution_spec.ns)

    @property
    def coupling_matrix_shape(self):
        return (self._model_spec.ncm, self._execution_spec.ups, self._execution_spec.ns,
                self._execution_spec.tile)

    @property
    def control_param_shape(self):
        return (self._model_spec.ncp, self._execution_spec.ns)

    @property
    def dense_state_shape(self):
        return (self._execution_spec.ndo, self._model_spec.sd, self._execution_spec.ns,
                self._execution_spec.tile)

    @property
    def dense_time_shape(self):
        return (self._execution_spec.ndo, self._execution_spec.ns)

    @property
    def dense_index_shape(self):
        return (self._execution_spec.ns,)

    @property
    def status_buffer_shape(self):
        return (self._execution_spec.ns,)

    # ---- solve (reference model.py:108-162) ----
    def solve(self, max_steps: int = 100_000, kernel_steps: int = 2048, *,
              sync_to_host: bool = False, sync_from_host: bool = False, stream=None,
              benchmark: bool = False, debug: bool = False):
        self._ensure_buffers()
        rt = self.runtime
        if sync_from_host:
            self.buffer_ops.sync_to_device(rt.host_buffers.state, rt.device_buffers.state, stream)
            self.buffer_ops.sync_to_device(rt.host_buffers.dense, rt.device_buffers.dense, stream)
        if rt.solver is None:
            rt.solver = self._make_solver(rt.backend, rt.variant)
        out = rt.solver(d_buffers=rt.device_buffers, model_spec=self._model_spec,
                        execution_spec=self._execution_spec, solver_spec=self._solver_spec,
                        max_steps=max_steps, kernel_steps=kernel_steps, benchmark=benchmark,
                        debug=debug)
        if sync_to_host:
            self.buffer_ops.sync_to_host(rt.device_buffers.state, rt.host_buffers.state, stream)
            self.buffer_ops.sync_to_host(rt.device_buffers.dense, rt.host_buffers.dense, stream)
            self.buffer_ops.sync_to_host(rt.device_buffers.status, rt.host_buffers.status, stream)
        return out

    def build_parameters(self):
        raise NotImplementedError

    def build_control_parameters(self):
        raise NotImplementedError

    def build_default_initial_state(self):
        raise NotImplementedError

    # ---- host buffers (reference model.py:180-225) ----
    def _initialize_host_buffers(self) -> None:
        unit_params, system_params, coupling_matrices = self.build_parameters()
        control_params = self.build_control_parameters()
        params = ParameterBuffer(unit_params=unit_params, system_params=system_params,
                                 control_params=control_params, coupling_matrices=coupling_matrices)
        state = ActualStateBuffer(
            actual_time=np.zeros(self.time_shape, dtype=np.float64),
            time_end=np.ones(self.time_shape, dtype=np.float64),
            time_begin=np.zeros(self.time_shape, dtype=np.float64),
            time_step=np.full(self.time_shape, 1e-6, dtype=np.float64),
            actual_state=self.build_default_initial_state(),
        )
        dense = DenseOutputBuffer(
            dense_index=np.zeros(self.dense_index_shape, dtype=np.int32),
            dense_time=np.zeros(self.dense_time_shape, dtype=np.float64),
            dense_state=np.zeros(self.dense_state_shape, dtype=np.float64),
        )
        status = StatusBuffer(
            # -1: "not initialised", must not be 0 or the event test would stop the system
            actual_event=np.full(self.status_buffer_shape, -1.0, dtype=np.float64),
            status_flags=np.zeros(self.status_buffer_shape, dtype=np.int32),
            total_steps=np.zeros(self.status_buffer_shape, dtype=np.int32),
            rejected_steps=np.zeros(self.status_buffer_shape, dtype=np.int32),
            convergece_success=np.zeros(self.status_buffer_shape, dtype=np.int32),
            convergence_failures=np.zeros(self.status_buffer_shape, dtype=np.int32),
        )
        self.runtime.host_buffers = BufferSet(state=state, params=params, dense=dense, status=status)

    def _ensure_buffers(self, stream=None) -> None:
        if self.runtime.device_buffers is not None:
            return
        hb = self.runtime.host_buffers
        ops = self.buffer_ops
        self.runtime.device_buffers = BufferSet(
            state=ops.create_device_state(hb.state), params=ops.create_device_params(hb.params),
            dense=ops.create_device_dense_output(hb.dense), status=ops.create_device_status(hb.status))

    # ---- shape checks (reference model.py:241-279) ----
    def _check_shape(self, x: np.ndarray, expected: tuple, name: str) -> None:
        if x.shape != expected:
            raise ValueError(f"{name} shape mismatch: expected {expected}, got {x.shape}")

    def _shape_check_all(self, R0, FREQ, PA, PS) -> None:
        ns = self._execution_spec.ns
        ups = self._execution_spec.ups
        tile = self._execution_spec.tile
        nk = self._model_spec.nk
        R0 = np.asarray(R0, dtype=np.float64)
        FREQ = np.asarray(FREQ, dtype=np.float64)
        PA = np.asarray(PA, dtype=np.float64)
        PS = np.asarray(PS, dtype=np.float64)
        if R0.ndim != 2:
            raise ValueError(f"R0 must be 2D with shape ({ns}, {ups}) or ({ns}, {tile}), got {R0.shape}")
        if FREQ.ndim != 2:
            raise ValueError(f"FREQ must be 2D with shape ({nk}, {ns}), got {FREQ.shape}")
        if PA.ndim != 2:
            raise ValueError(f"PA must be 2D with shape ({nk}, {ns}), got {PA.shape}")
        if PS.ndim != 2:
            raise ValueError(f"PS must be 2D with shape ({nk}, {ns}), got {PS.shape}")
        if R0.shape not in ((ns, ups), (ns, tile)):
            raise ValueError(f"R0 shape mismatch: expected ({ns}, {ups}) or already padded ({ns}, {tile}), "
                             f"got {R0.shape}")
        for arr, nm in ((FREQ, "FREQ"), (PA, "PA"), (PS, "PS")):
            if arr.shape != (nk, ns):
                raise ValueError(f"{nm} shape mismatch: expected {(nk, ns)}, got {arr.shape}")

    def _make_solver(self, b: BackendName, v: KernelVariant) -> Callable[..., Any]:
        raise NotImplementedError
