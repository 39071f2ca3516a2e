"""Compile-option record accepted by ``CKM1D(...)``.

Same fields and mode semantics as ``coupledbubble_control/backends/cuda_opts.py``
(:6-73).  The B200 library is built ahead of time for sm_100a, so nothing
reads this record: ``CKM1D(...)`` stores it only so that constructors written
for the reference (``compiler=``, ``max_registers=``, ``fastmath=``,
``cuda_mode=``) keep working unchanged.
"""
from dataclasses import dataclass
from typing import Literal, Optional


@dataclass
class CUDAOpts:
    mode: Literal["debug", "profile", "release"] = "release"
    max_registerts: Optional[int] = None      # (sic) field name of the reference
    fastmath: bool = False
    lineinfo: bool = False
    opt: bool = True
    debug: bool = False
    cache: bool = False
    xptxas_verbose: bool = False
    warn_spills: bool = False
    compiler: Literal["nvrtc", "nvcc"] = "nvrtc"

    def __post_init__(self):
        if self.mode == "debug":
            self.debug = True
            self.lineinfo = True
            self.xptxas_verbose = True
            self.warn_spills = True
        elif self.mode == "profile":
            self.debug = False
            self.lineinfo = True
            self.xptxas_verbose = True
            self.warn_spills = True
        elif self.mode == "release":
            self.debug = False
            self.lineinfo = False
            self.xptxas_verbose = False
            self.warn_spills = False
            self.fastmath = False
