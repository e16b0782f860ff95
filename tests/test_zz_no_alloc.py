"""fireCudaForceProjectNoAlloc against the regular force pass (needs a GPU).

The allocation-free entry point serves callers that cannot let the library
call cudaMalloc: engines that own all device memory, frames captured into CUDA
graphs, hosts that forbid allocations after start-up.  Here the caller's
buffers are torch tensors; the entry point only queues the force kernels on the
caller's stream and keeps its per-cell increments in the library's fixed
scratch array.  Its outputs must equal those of the regular path
(fireCudaRunStages FORCE..DIVERGENCE on the same state), on two calls in a row.
This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import tolerances as T

pytestmark = pytest.mark.gpu


def _no_alloc_fn(pkg, precision="f32"):
    lib = pkg.load_library(precision)
    fn = lib.fireCudaForceProjectNoAlloc
    fn.restype = ctypes.c_bool
    fn.argtypes = [ctypes.POINTER(pkg.abi.FireSettings), ctypes.c_float] + [ctypes.c_int] * 3 + [ctypes.c_void_p] * 12
    return fn


def _call(fn, pkg, settings, time, dims, inputs, outputs, stream):
    nx, ny, nz = dims
    ok = fn(ctypes.byref(settings), time, nx, ny, nz, *[ctypes.c_void_p(t.data_ptr()) for t in inputs],
            *[ctypes.c_void_p(t.data_ptr()) for t in outputs], ctypes.c_void_p(stream))
    assert ok, pkg.firesim.last_error()


STORAGE = {"f32": "float32", "f16": "float16", "bf16": "bfloat16"}


@pytest.mark.parametrize("precision", ["f32", "f16", "bf16"])
def test_no_alloc_force_pass_matches_regular_path(pkg, abi, precision):
    """Each library build takes records and faces in its own storage type."""
    import torch

    fn = _no_alloc_fn(pkg, precision)
    storage = getattr(torch, STORAGE[precision])
    dims = (40, 48, 32)
    sim = pkg.FireSim(64, 40, *dims, precision=precision)
    stream = torch.cuda.current_stream().cuda_stream
    for frame in range(2):
        # Advance the scene so the force pass sees a developed fire.
        for f in range(4 * frame, 4 * frame + 4):
            sim.step(abi.validation_settings(f, width=64, height=40))
        sim.synchronize()
        settings = abi.validation_settings(4 * frame + 4, width=64, height=40)
        time = float(np.float32(sim.times()[0]) + np.float32(settings.dt))
        f = {n: sim.get(n) for n in abi.SCALAR_FIELDS + ["u", "v", "w"]}
        # The scene's fields come back as float; in the half builds they hold
        # stored half values, so converting back to the storage type is exact.
        rec_a = torch.tensor(np.stack([f["heat"], f["fuel"], f["oxygen"], f["soot"]], axis=-1), device="cuda").to(storage)
        rec_b = torch.tensor(np.stack([f["char"], f["ash"], f["pyrolysis"], f["progress"]], axis=-1), device="cuda").to(storage)
        rec_c = torch.tensor(np.stack([f["turbulence_energy"], f["soot_optics"]], axis=-1), device="cuda").to(storage)
        faces = [torch.tensor(f[n], device="cuda").to(storage) for n in ("u", "v", "w")]
        outs = [torch.full_like(t, np.nan) for t in faces]
        div = torch.full(f["heat"].shape, np.nan, device="cuda")
        pres = torch.full(f["heat"].shape, np.nan, device="cuda")
        _call(fn, pkg, settings, time, dims, [rec_a, rec_b, rec_c, *faces], [*outs, div, pres], stream)
        torch.cuda.synchronize()
        outs = [t.float() for t in outs]

        sim.stages("force", "divergence", settings, time)
        expect = {n: sim.get(n) for n in ("u", "v", "w", "divergence", "pressure")}
        got = {"u": outs[0], "v": outs[1], "w": outs[2], "divergence": div, "pressure": pres}
        for n, ref in expect.items():
            T.check_field(f"call{frame}/{n}", got[n].cpu().numpy(), ref, T.GPU_EXACT)
    sim.close()


def test_no_alloc_rejects_oversized_grid(pkg, abi):
    import torch

    fn = _no_alloc_fn(pkg)
    dummy = torch.zeros(16, device="cuda")
    settings = abi.FireSettings()
    ok = fn(ctypes.byref(settings), 0.0, 128, 128, 128, *[ctypes.c_void_p(dummy.data_ptr())] * 11,
            ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(0))
    assert not ok
    assert "exceeds the 1048576-cell scratch" in pkg.firesim.last_error()
    ok = fn(ctypes.byref(settings), 0.0, 2, 2, 70000, *[ctypes.c_void_p(dummy.data_ptr())] * 11,
            ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(0))
    assert not ok
    assert "at most 65535" in pkg.firesim.last_error()
