"""Backend selector of the CKM1D model.

Mirrors ``coupledbubble_control/backends/__init__.py:4-10`` and adds one
member, ``B200``, which routes ``Model.solve`` to the sm_100a library through
its C ABI (``include/cbc_b200.h``).  The reference's ``cupy``/``numba`` names
are kept so that code selecting them still parses; only ``B200`` is served by
this package.
"""
from enum import Enum

from .cuda_opts import CUDAOpts


class BackendName(str, Enum):
    CUPY = "cupy"
    NUMBA = "numba"
    B200 = "b200"


class KernelVariant(str, Enum):
    WARP = "warp"
    SHARED = "shared"


def get_current_device_name() -> str:
    """Sanitised CUDA device name, e.g. ``B200`` (reference backends/__init__.py:13-39)."""
    import re
    try:
        import torch
        name = torch.cuda.get_device_name()
    except Exception:
        return "unknownGPU"
    name = re.sub(r"[^a-zA-Z0-9]", "", name)
    return name.replace("NVIDIA", "").replace("GeForce", "")


__all__ = ["BackendName", "KernelVariant", "CUDAOpts", "get_current_device_name"]
