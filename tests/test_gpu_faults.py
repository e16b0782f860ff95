"""Host-side failure injection of device allocations (needs a GPU for the
library's context; nothing faults on the GPU: the failing cudaMalloc is never
made).  An initialisation that runs out of memory fails with the reference's
error convention ("label: error string", src/fire_cuda.cu:197-207), frees
what it had allocated (src/fire_cuda.cu:2981) and leaves the library usable.
"""
from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_allocation_failure_is_reported_freed_and_recovered(pkg, abi):
    import torch

    lib = pkg.load_library()
    sim = pkg.FireSim(64, 48, 32, 32, 32)  # a first context and scene, so later figures are steady
    sim.close()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for succeed in (0, 1, 5, 17):
        assert lib.fireCudaSetAllocationFault(succeed)
        assert not lib.fireCudaInitializeGrid(64, 48, 32, 32, 32)
        msg = pkg.firesim.last_error()
        assert "out of memory (injected)" in msg and ": " in msg, msg
        dims = (ctypes.c_int * 8)()
        assert not lib.fireCudaGetGridInfo(dims)  # no scene after a failed init
        assert "not initialized" in pkg.firesim.last_error()
    assert lib.fireCudaSetAllocationFault(-1)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after >= free_before - (64 << 20), (free_before, free_after)
    sim = pkg.FireSim(64, 48, 32, 32, 32)
    sim.step(abi.validation_settings(0, width=64, height=48))
    sim.synchronize()
    assert sim.get("heat").sum() > 0.0
    sim.close()


def test_scene_handle_allocation_failure(pkg, abi):
    lib = pkg.load_library()
    assert lib.fireCudaSetAllocationFault(2)
    try:
        with pytest.raises(pkg.FireSimError, match="out of memory"):
            pkg.Scene(32, 16, 24, 24, 24)
    finally:
        assert lib.fireCudaSetAllocationFault(-1)
    sc = pkg.Scene(32, 16, 24, 24, 24)
    sc.close()
    assert not lib.fireCudaSetAllocationFault(-2)
