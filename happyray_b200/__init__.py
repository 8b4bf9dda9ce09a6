"""happyray_b200: B200-native grid build + grid traversal (drop-in for the javorkk/happyray hot path).

The compute path is libhappyray_b200.so (hand-written sm_100a CUDA kernels behind the
C-ABI in include/happyray.h).  This package holds the host-side mirror of the
reference's RTEngine interface (engine.Engine), the ctypes binding (_lib) and the
seeded synthetic scene generators used by the tests and the bench (scenes).
"""
from ._lib import (GRID_TWO_LEVEL, GRID_UNIFORM, RENDER_AO, RENDER_PATH, RENDER_PATH_SINGLE_KERNEL,  # noqa: F401
                   RENDER_PRIMARY, HRError, load)
from .engine import Engine  # noqa: F401

__all__ = ["Engine", "HRError", "load", "GRID_UNIFORM", "GRID_TWO_LEVEL", "RENDER_PRIMARY", "RENDER_PATH",
           "RENDER_PATH_SINGLE_KERNEL", "RENDER_AO"]
