"""B200 (sm_100a) implementation of the LePIC per-timestep PIC-MCC loop.

The compute path is the in-tree CUDA library ``_lib/liblepic_gpu.so`` behind the C ABI of
``include/lepic_gpu.h``; this package is its host side (decks, configurations, the step
driver) and has no CPU fallback for any hot routine.
"""
from . import _capi, configs, deck  # noqa: F401

__all__ = ["_capi", "configs", "deck", "GpuSimulation", "build_library"]


def build_library(force: bool = False) -> str:
    from .build import build
    return build(force=force)


def __getattr__(name):
    if name == "GpuSimulation":
        from .simulation import GpuSimulation
        return GpuSimulation
    raise AttributeError(name)
