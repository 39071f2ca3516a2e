from .ckm1d import CKM1D
from .model import MaterialProperties, water
from .specs import ExecutionSpec, LayoutEntry, ModelSpec, SolverSpec

__all__ = ["CKM1D", "MaterialProperties", "water", "ModelSpec", "ExecutionSpec", "SolverSpec",
           "LayoutEntry"]
