from .pos_control import CKM1DVecEnv, SceneGenerator

__all__ = ["CKM1DVecEnv", "SceneGenerator"]
