"""B200-native CKM1D ensemble integrator.

Host-side mirror of the reference's ``coupledbubble_control`` model API
(models, backends) in front of an sm_100a CUDA library reached through a C ABI
(``include/cbc_b200.h``).  There is no CPU fallback: every solve runs on the
GPU, and importing the solver without the built library raises.
"""
from .backends import BackendName, KernelVariant
from .models import CKM1D, MaterialProperties, SolverSpec, water

__all__ = ["BackendName", "KernelVariant", "CKM1D", "MaterialProperties", "SolverSpec", "water"]
