"""firesim-b200: a B200-native (sm_100a) rewrite of native-firesim's per-frame volume pipeline.

The product is the shared library native-firesim_b200/libfiresim_b200.so, whose
C ABI is declared in include/fire_cuda.h (the reference's seventeen entry
points) and include/fire_ext.h (grid-explicit scenes, field access, stages,
batching).  This Python package is a thin ctypes binding over that ABI for
tests, benchmarks and Python callers; it performs no computation itself.
"""
from __future__ import annotations

from . import abi  # noqa: F401
from .firesim import (Batch, FireSim, FireSimError, Scene, Server, batch_step, check_guards, load_library, set_autotune,  # noqa: F401
                      tuned_brick)

__all__ = ["abi", "Batch", "FireSim", "FireSimError", "Scene", "Server", "batch_step", "check_guards", "load_library", "set_autotune", "tuned_brick"]
