"""Frozen specification records of the CKM1D integrator.

Same fields, defaults and validation as the reference's
``coupledbubble_control/models/specs.py`` (ModelSpec :6-23, ExecutionSpec
:27-52, SolverSpec :56-72, LayoutEntry :75-79), so code written against the
reference constructs them unchanged.  Fields added here (``dense_mode``,
``col_threshold``) have defaults that reproduce the reference behaviour.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Literal


@dataclass(frozen=True)
class ModelSpec:
    name: str           # model name
    sd: int             # state components per bubble
    nup: int            # per-bubble parameters
    nsp: int            # per-system parameters
    ncm: int            # coupling matrices
    nk: int             # harmonic components of the drive
    ne: int             # events
    ncf: int            # coupling factors
    nct: int            # coupling terms
    ac: Literal["CONST", "SW_N", "SW_A"]
    ncp: int = field(init=False)   # 4 * nk control parameters (PA, omega, phase, wave number)

    def __post_init__(self) -> None:
        object.__setattr__(self, "ncp", 4 * self.nk)


@dataclass(frozen=True)
class ExecutionSpec:
    ups: int          # bubbles ("units") per system
    ns: int = 1       # systems
    spb: int = 1      # systems per block (kept for API compatibility; the B200 kernels pick their own)
    ndo: int = 0      # dense-output samples per system (0: none)

    tile: int = field(init=False)            # ups padded to a power of two (row width of the buffers)
    total_threads: int = field(init=False)
    active_threads: int = field(init=False)
    block_size: int = field(init=False)
    grid_size: int = field(init=False)

    def __post_init__(self) -> None:
        if self.ups < 1:
            raise ValueError("ups must be > 1")
        if self.ns < 1:
            raise ValueError("ns must be >= 1")
        if self.spb < 1:
            raise ValueError("spb must be >= 1")
        object.__setattr__(self, "tile", 1 << (self.ups - 1).bit_length())
        object.__setattr__(self, "total_threads", self.ns * self.tile)
        object.__setattr__(self, "active_threads", self.ns * self.ups)
        object.__setattr__(self, "block_size", self.spb * self.tile)
        object.__setattr__(self, "grid_size", (self.ns + self.spb - 1) // self.spb)


@dataclass(frozen=True)
class SolverSpec:
    # ODE solver
    atol: float = 1e-9
    rtol: float = 1e-9
    min_step: float = 1e-16
    max_step: float = 1e-1
    growth_limit: float = 2.0     # present in the reference, unused by its kernels
    shrink_limit: float = 0.5     # present in the reference, unused by its kernels
    # implicit coupling (relaxed Richardson)
    lin_atol: float = 1e-9
    lin_rtol: float = 1e-9
    lin_max_iter: int = 100
    lin_relaxation: float = 2.0 / 3.0
    etol: float = 1.0e-5
    # additions (defaults reproduce the reference kernels)
    col_threshold: float = 0.1            # collision gap factor is (1 + col_threshold)
    dense_mode: Literal["reference", "grid"] = "reference"
    # implicit-coupling solver: "richardson" (the reference's relaxed
    # iteration, lin_* fields above) or "lu" (direct solve by Gauss-Jordan
    # elimination with partial pivoting; exact to rounding, never iterates)
    lin_solver: Literal["richardson", "lu"] = "richardson"

    def __post_init__(self):
        if self.lin_solver not in ("richardson", "lu"):
            raise ValueError(f"lin_solver must be 'richardson' or 'lu', got {self.lin_solver!r}")


@dataclass(frozen=True)
class LayoutEntry:
    group: str
    base_offset: int
