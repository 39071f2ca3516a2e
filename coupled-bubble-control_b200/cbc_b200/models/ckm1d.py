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

    # ---- parameter precompute (reference ckm1d.py:133-202) ----
    def build_parameters(self):
        unit_params = np.zeros(self.unit_param_shape, dtype=np.float64)
        system_params = np.zeros(self.system_param_shape, dtype=np.float64)
        coupling_matrices = np.zeros(self.coupling_matrix_shape, dtype=np.float64)
        ups = self._execution_spec.ups
        c = precompute_constants(self.mat_props, self._REF_FREQ)
        R0 = self._R0[:, :ups]
        unit_params[:, :, :ups] = bubble_constants(R0, c)
        system_params[:] = np.asarray(system_constants(c))[:, None]
        # coupling_matrices[m, j, s, i]: source bubble j, receiving bubble i
        cm = coupling_constants(R0, c)                       # (3, ns, j, i)
        coupling_matrices[:, :ups, :, :ups] = np.transpose(cm, (0, 2, 1, 3))
        return unit_params, system_params, coupling_matrices

    def build_control_parameters(self):
        control_params = np.zeros(self.control_param_shape, dtype=np.float64)
        nk = self._model_spec.nk
        c = precompute_constants(self.mat_props, self._REF_FREQ)
        control_params[0:nk, :] = self._PA
        control_params[nk:2 * nk, :] = self._FREQ * c["two_pi"]
        control_params[2 * nk:3 * nk, :] = self._PS
        control_params[3 * nk:4 * nk, :] = c["two_pi"] * self._FREQ / c["CL"]
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


# ---- the precompute as array formulas over the radii -----------------------
# The same arithmetic as the reference's build_parameters
# (models/ckm1d.py:133-188) and build_control_parameters (:190-202), written
# as products and quotients of per-bubble arrays and scalar constants so that
# the device precompute (csrc/admit.cu) can repeat it operation for operation.
# The one deliberate difference: cubes are (x * x) * x instead of numpy's
# x ** 3 (a libm pow call, which a GPU cannot reproduce bit for bit); the two
# differ by at most an ulp.

def precompute_constants(mp, ref_freq_hz: float) -> dict:
    """Scalar constants of the precompute (Python floats, host-evaluated)."""
    two_pi = 2.0 * np.pi
    w_ref = two_pi * ref_freq_hz
    l_ref = mp.CL / ref_freq_hz
    return {
        "two_pi": two_pi, "w_ref": w_ref, "l_ref": l_ref,
        "RHO": mp.RHO, "CL": mp.CL, "P0": mp.P0, "PV": mp.PV, "PE": mp.PE, "ST": mp.ST, "VIS": mp.VIS,
        "st2": 2.0 * mp.ST,                           # 2 sigma
        "k1": 1.0 - 3.0 * mp.PE,                      # 1 - 3 gamma
        "p0pv": mp.P0 - mp.PV,
        "k4": 4.0 * mp.VIS / mp.RHO,
        "tw": two_pi / w_ref,                         # 2 pi / omega_ref
        "k6": ((two_pi / w_ref) ** 2.0) / mp.CL / mp.RHO,
        "hl": 0.5 * l_ref,
        "k9": two_pi / mp.RHO,
        "k10": 2 * two_pi / 3,
        "k11": 6 * two_pi * mp.VIS,
        "km2": (18 * mp.VIS / mp.RHO) * (two_pi / w_ref),
    }


def bubble_constants(R0: np.ndarray, c: dict) -> np.ndarray:
    """The 13 per-bubble constants (unit_params) of radii R0 (m), any shape:
    result shape (13,) + R0.shape."""
    R0 = np.asarray(R0, dtype=np.float64)
    s = c["two_pi"] / R0 / c["w_ref"]
    s2 = s * s
    pe = c["st2"] / R0 + c["P0"] - c["PV"]
    q = c["hl"] / R0
    wr = c["w_ref"] * R0
    out = np.empty((13,) + R0.shape)
    # Keller--Miksis
    out[0] = pe * s2 / c["RHO"]
    out[1] = c["k1"] * pe * s / c["CL"] / c["RHO"]
    out[2] = c["p0pv"] * s2 / c["RHO"]
    out[3] = (c["st2"] / R0 / c["RHO"]) * s2
    out[4] = c["k4"] / (R0 * R0) * c["tw"]
    out[5] = s2 / c["RHO"]
    out[6] = c["k6"] / R0
    out[7] = R0 * c["w_ref"] / c["two_pi"] / c["CL"]
    # translational motion
    out[8] = q * q
    out[9] = c["k9"] / R0 / c["l_ref"] / (wr * wr)
    out[10] = c["k10"] * ((R0 * R0) * R0)
    out[11] = c["k11"] * R0
    out[12] = R0 / c["l_ref"]
    return out


def system_constants(c: dict):
    """The 5 per-system constants (system_params)."""
    return [3.0 * c["PE"], 1.0 / c["w_ref"], c["l_ref"] / c["two_pi"], c["CL"], 1 / c["RHO"] / c["CL"]]


def coupling_constants(R0: np.ndarray, c: dict) -> np.ndarray:
    """Coupling coefficients of systems with radii R0 (ns, K) in metres:
    (3, ns, K, K) indexed [m, s, j, i] (source bubble j, receiving bubble i),
    zero for j == i."""
    R0 = np.asarray(R0, dtype=np.float64)
    Rj = R0[:, :, None]                   # source
    Ri = R0[:, None, :]                   # receiver
    rl = Rj / c["l_ref"]
    out = np.empty((3,) + Rj.shape[:2] + (R0.shape[1],))
    out[0] = ((Rj * Rj) * Rj) / (Ri * Ri) / c["l_ref"]
    out[1] = 3.0 * ((rl * rl) * rl)
    out[2] = c["km2"] * ((rl * rl) * rl) / (Ri * Ri)
    K = R0.shape[1]
    idx = np.arange(K)
    out[:, :, idx, idx] = 0.0             # no self coupling
    return out
