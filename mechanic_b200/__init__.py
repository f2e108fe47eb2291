"""mechanic_b200 — B200-native (sm_100a) rigid-body step of jens-hj/mechanic.

The compute path is libmechanic_b200.so (hand-written CUDA behind a C ABI,
include/mechanic_b200.h).  Python here only mirrors the reference's
``GpuPhysics`` interface over that ABI and generates seeded scenes.
"""
from . import abi, scenes  # noqa: F401

__all__ = ["abi", "scenes", "physics", "ops"]


def __getattr__(name):
    # physics/ops load the CUDA library lazily: importing the package never
    # needs a GPU, calling into it does (and fails loudly without the .so).
    if name in ("physics", "ops"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    if name in ("GpuPhysics", "GpuPhysicsConfig"):
        from . import physics
        return getattr(physics, name)
    raise AttributeError(name)
