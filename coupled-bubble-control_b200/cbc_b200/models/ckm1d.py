"""Coupled Keller--Miksis bubble model with 1D translational motion (CKM1D).

Mirrors ``coupledbubble_control/models/ckm1d.py``: the constructor
(:32-130, same arguments and unit conversions: um, bar, kHz, PS in units of
pi), the parameter precompute ``build_parameters`` (:133-188) and
``build_control_parameters`` (:190-202), the default initial state
(:204-212) and ``_make_solver`` (:214-253), which here serves
``BackendName.B200`` through the C ABI of the sm_100a library.
"""
from __future__ import annotations

from typing import Any, Callable, Literal, Optional

import numpy as np

from .model import MaterialProperties, Model, ModelRuntime
from .specs import ExecutionSpec, LayoutEntry, ModelSpec, SolverSpec
from .buffers import BufferOps
from ..backends import BackendName, CUDAOpts, KernelVariant


class CKM1D(Model):
    _available_backends = (BackendName.B200,)
    _kernel_variants = (KernelVariant.SHARED, KernelVariant.WARP)

    def __init__(self, num_systems: int, systems_per_block: int, units_per_system: int,
                 R0, PA, FR, PS, REF_FREQ: float = 20.0, num_components: int = 2,
                 acoustic_field: Literal["CONST", "SW_N", "SW_A"] = "CONST",
                 mat_props: Optional[MaterialProperties] = None,
                 backend: BackendName = BackendName.B200,
                 variant: KernelVariant = KernelVariant.SHARED,
                 num_stored_points: int = 0,
                 compiler: Literal["nvrtc", "nvcc"] = "nvcc",
                 max_registers: Optional[int] = None, fastmath: bool = True,
                 cuda_mode: Literal["debug", "profile", "release"] = "release",
                 solver_spec: Optional[SolverSpec] = None,
                 verbose: bool = False) -> None:
        self._model_spec = ModelSpec(name="CKM1D", sd=4, nup=13, nsp=5, ncm=3, ne=1, ncf=4, nct=8,
                                     nk=num_components, ac=acoustic_field)
        self._execution_spec = ExecutionSpec(ns=num_systems, spb=systems_per_block,
                                             ups=units_per_system, ndo=num_stored_points)
        self._cuda_opts = CUDAOpts(mode=cuda_mode, fastmath=fastmath, max_registerts=max_registers,
                                   compiler=compiler)
        self._solver_spec = solver_spec if solver_spec is not None else SolverSpec()
        backend = BackendName(backend)
        self.runtime = ModelRuntime(backend, KernelVariant(variant))
        self.buffer_ops = BufferOps(backend)
        self.control_layout = {
            "PA": LayoutEntry("control_params", 0),
            "FR": LayoutEntry("control_params", num_components),
            "PS": LayoutEntry("control_params", 2 * num_components),
            "WL": LayoutEntry("control_params", 3 * num_components),
        }
        self.state_layout = {
            "R": LayoutEntry("actual_state", 0),
            "X": LayoutEntry("actual_state", 1),
            "U": LayoutEntry("actual_state", 2),
            "V": LayoutEntry("actual_state", 3),
        }
        self.mat_props = mat_props if mat_props is not None else MaterialProperties()
        self._shape_check_all(R0, FR, PA, PS)
        # SI units (reference ckm1d.py:114-117)
        self._REF_FREQ = REF_FREQ * 1000.0
        self._FREQ = np.ascontiguousarray(FR, dtype=np.float64) * 1000.0
        self._PA = np.ascontiguousarray(PA, dtype=np.float64) * 1.0e5
        self._PS = np.ascontiguousarray(PS, dtype=np.float64) * np.pi
        ns, tile, ups = self._execution_spec.ns, self._execution_spec.tile, self._execution_spec.ups
        R0 = np.asarray(R0, dtype=np.float64)
        if R0.shape == (ns, tile):
            self._R0 = np.ascontiguousarray(R0) * 1.0e-6
        else:
            self._R0 = np.zeros((ns, tile), dtype=np.float64)
            self._R0[:, :ups] = R0 * 1e-6
        if verbose:
            print("Padding Applied" if R0.shape != (ns, tile) else "NO Padding Applied (already padded)")
        self._initialize_host_buffers()

    # ---- parameter precompute (reference ckm1d.py:133-188) ----
    def build_parameters(self):
        unit_params = np.zeros(self.unit_param_shape, dtype=np.float64)
        system_params = np.zeros(self.system_param_shape, dtype=np.float64)
        coupling_matrices = np.zeros(self.coupling_matrix_shape, dtype=np.float64)
        TWO_PI = 2.0 * np.pi
        mp = self.mat_props
        PV, RHO, ST, VIS, CL, P0, PE = mp.PV, mp.RHO, mp.ST, mp.VIS, mp.CL, mp.P0, mp.PE
        UPS = self._execution_spec.ups
        w_ref = TWO_PI * self._REF_FREQ
        l_ref = CL / self._REF_FREQ
        R0 = self._R0[:, :UPS]
        # Keller--Miksis
        unit_params[0, :, :UPS] = (2.0 * ST / R0 + P0 - PV) * (TWO_PI / R0 / w_ref) ** 2.0 / RHO
        unit_params[1, :, :UPS] = (1.0 - 3.0 * PE) * (2 * ST / R0 + P0 - PV) * (2.0 * np.pi / R0 / w_ref) / CL / RHO
        unit_params[2, :, :UPS] = (P0 - PV) * (2.0 * np.pi / R0 / w_ref) ** 2.0 / RHO
        unit_params[3, :, :UPS] = (2.0 * ST / R0 / RHO) * (TWO_PI / R0 / w_ref) ** 2.0
        unit_params[4, :, :UPS] = 4.0 * VIS / RHO / (R0 ** 2.0) * (2.0 * np.pi / w_ref)
        unit_params[5, :, :UPS] = ((2.0 * np.pi / R0 / w_ref) ** 2.0) / RHO
        unit_params[6, :, :UPS] = ((2.0 * np.pi / w_ref) ** 2.0) / CL / RHO / R0
        unit_params[7, :, :UPS] = R0 * w_ref / (2 * np.pi) / CL
        # translational motion
        unit_params[8, :, :UPS] = (0.5 * l_ref / R0) ** 2
        unit_params[9, :, :UPS] = TWO_PI / RHO / R0 / l_ref / (w_ref * R0) ** 2.0
        unit_params[10, :, :UPS] = 2 * TWO_PI / 3 * R0 ** 3
        unit_params[11, :, :UPS] = 6 * TWO_PI * VIS * R0
        unit_params[12, :, :UPS] = R0 / l_ref
        # shared
        system_params[0] = 3.0 * PE
        system_params[1] = 1.0 / w_ref
        system_params[2] = l_ref / TWO_PI
        system_params[3] = CL
        system_params[4] = 1 / RHO / CL
        # coupling matrices, row = source bubble j, last axis = receiving bubble i
        l_ref_mx = np.full_like(R0, l_ref)
        for row in range(UPS):
            coupling_matrices[0, row, :, :UPS] = R0[:, row:row + 1] ** 3 / R0 ** 2 / l_ref
            coupling_matrices[1, row, :, :UPS] = 3.0 * (R0[:, row:row + 1] / l_ref_mx) ** 3
            coupling_matrices[2, row, :, :UPS] = (18 * VIS / RHO) * (TWO_PI / w_ref) * (R0[:, row:row + 1] / l_ref) ** 3 / (R0 ** 2)
        idx = np.arange(UPS)
        coupling_matrices[:, idx, :, idx] = 0.0   # no self coupling
        return unit_params, system_params, coupling_matrices

    def build_control_parameters(self):
        control_params = np.zeros(self.control_param_shape, dtype=np.float64)
        TWO_PI = 2.0 * np.pi
        CL = self.mat_props.CL
        NC = self._model_spec.nk
        control_params[0:NC, :] = self._PA
        control_params[NC:2 * NC, :] = self._FREQ * TWO_PI
        control_params[2 * NC:3 * NC, :] = self._PS
        control_params[3 * NC:4 * NC, :] = TWO_PI * self._FREQ / CL
        return control_params

    def build_default_initial_state(self):
        state = np.zeros(self.state_shape, dtype=np.float64)
        ups = self._execution_spec.ups
        state[0, :, :ups] = 1.0
        return state

    # ---- solver selection (reference ckm1d.py:214-253) ----
    def _make_solver(self, b: BackendName, v: KernelVariant = KernelVariant.SHARED) -> Callable[..., Any]:
        from functools import partial
        if b == BackendName.B200:
            from ..backends.b200_solver import load_kernel, solver
            kernel = load_kernel(self._model_spec, self._execution_spec, self._solver_spec)
            return partial(solver, kernel=kernel)
        raise NotImplementedError(f"backend {b!r} is not served by this package (use BackendName.B200)")
