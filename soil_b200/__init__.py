"""soil_b200 — B200-native (sm_100a) substrate hot path of SOIL.

The compute path is the CUDA library ``libsoil_cuda.so`` (C ABI declared in
include/soil_cuda.h).  ``System`` is its Python binding; ``workloads`` builds
the seeded synthetic inputs.
"""
from . import abi  # noqa: F401


def __getattr__(name):
    if name in ("System", "Context"):
        from . import system
        return getattr(system, name)
    raise AttributeError(name)
