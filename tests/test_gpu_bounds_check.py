"""The bounds-checking build, libfiresim_b200_checked.so (-DFIRE_BOUNDS_CHECK),
on the GPU.

In that build every device buffer the library owns sits between two 2 MiB
guard zones, and the whole allocation starts as 0xFF bytes: NaN in every
float field, -1 in every integer.  A kernel that writes past either end of a
buffer changes a guard byte, which fireCudaCheckGuards reports by buffer
name; one that reads past an end, or reads a cell that nothing has written,
takes a NaN or a -1 into its result, so the checked build's fields and
frames would differ from the default build's.

Each workload runs on the checked build first, where a stray access stays
inside its allocation, and its guards are checked before the default build
runs the same workload for the bitwise comparison.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("heat", "fuel", "soot", "u", "v", "w", "pressure")


def _bits_equal(name, got, want):
    g, w = np.ascontiguousarray(got).view(np.uint32), np.ascontiguousarray(want).view(np.uint32)
    bad = int(np.count_nonzero(g != w))
    assert bad == 0, f"{name}: {bad}/{g.size} values differ"


def test_default_build_has_no_guards(pkg):
    assert pkg.check_guards("f32") == -1


def test_planted_guard_bytes_are_reported_once(pkg):
    """A byte set after the end of a live buffer (with a host-side memset inside
    its allocation) is named with its offset, then re-armed; one set in a
    buffer that is then freed is reported as freed."""
    sim = pkg.FireSim(32, 24, 24, 20, 16, precision="checked")
    lib = sim.lib
    try:
        assert pkg.check_guards() == 0
        assert lib.fireCudaPlantGuardByte(b"pressure", 5)
        with pytest.raises(pkg.FireSimError, match=r"'pressure' \(30720 bytes\): write past its end, first changed byte at end \+ 5$"):
            pkg.check_guards()
        assert pkg.check_guards() == 0
        # A 4-byte buffer: its end is not on a 16-byte boundary.
        assert lib.fireCudaPlantGuardByte(b"SOR status", 0)
        with pytest.raises(pkg.FireSimError, match=r"'SOR status' \(4 bytes\): write past its end, first changed byte at end \+ 0$"):
            pkg.check_guards()
        assert not lib.fireCudaPlantGuardByte(b"no such buffer", 0)
        assert lib.fireCudaPlantGuardByte(b"divergence", 1000)
    finally:
        sim.close()
    with pytest.raises(pkg.FireSimError, match=r"freed 'divergence' \(30720 bytes\): write past its end, first changed byte at end \+ 1000$"):
        pkg.check_guards()
    assert pkg.check_guards() == 0


@pytest.mark.parametrize("dims,path,scene", [((17, 21, 11), 0, 0), ((24, 20, 16), 1, 1), ((40, 34, 70), 0, 2)])
def test_reference_physics_keeps_guards_and_bits(pkg, abi, dims, path, scene):
    """Five frames of the reference physics (resident or colour-split SOR, a
    render every frame): no guard changes, and the fields and frames equal the
    default build's bit for bit."""
    runs = {}
    for precision in ("checked", "f32"):
        sim = pkg.FireSim(64, 48, *dims, precision=precision)
        sim.set_pressure_path(path)
        frames = []
        for f in range(5):
            s = abi.validation_settings(f, scene=scene, width=64, height=48)
            s.reset = 1 if f == 0 else 0
            frames.append(sim.step_and_render(s)[0])
        sim.synchronize()
        fields = {n: sim.get(n) for n in FIELDS}
        if precision == "checked":
            assert pkg.check_guards() == 0
        sim.close()
        if precision == "checked":
            assert pkg.check_guards() == 0
        runs[precision] = (fields, frames)
    (got, got_frames), (want, want_frames) = runs["checked"], runs["f32"]
    for n in FIELDS:
        _bits_equal(f"{dims}/{n}", got[n], want[n])
    for j, (g, w) in enumerate(zip(got_frames, want_frames)):
        _bits_equal(f"{dims}/frame{j}", g, w)
    assert want["heat"].sum() > 0.0


def _config_scene(pkg, abi, dims, k, precision):
    import torch

    nx, ny, nz = dims
    sc = pkg.Scene(48, 32, *dims, precision=precision)
    p = abi.config_scene(nx, ny, nz, nx / 2, nz / 2, max(2.0, min(nx, nz) / 5), 0.3, -0.2, 11 + k)
    p.pressureTop = 1
    sc.set_physics(p)
    sc.set_pressure_multigrid(20, 2, 2)
    sc.set_pressure_tolerance(1e-5, 1)
    hdr = torch.zeros((32, 48, 4), dtype=torch.float32, device="cuda")
    sc.set_hdr_buffer(hdr.data_ptr(), 48 * 16, 0)
    return sc, hdr


@pytest.mark.parametrize("dims", [(33, 17, 21), (125, 4, 99), (20, 36, 44)])
def test_config_multigrid_keeps_guards_and_bits(pkg, abi, dims):
    """Six steps of the config physics with the multigrid projection (a grid
    that coarsens unevenly, one that cannot coarsen in y, one whose tail does
    not start at 16^3), a render every third step: no guard changes, and the
    fields, frames and cycle counts equal the default build's."""
    runs = {}
    for precision in ("checked", "f32"):
        sc, hdr = _config_scene(pkg, abi, dims, 0, precision)
        frames, cycles = [], []
        for i in range(6):
            s = abi.FireSettings(width=48, height=32, dt=1.0 / 60.0)
            s.reset = 1 if i == 0 else 0
            sc.step(s, render=i % 3 == 2)
            cycles.append(sc.pressure_stats()[0])
            if i % 3 == 2:
                sc.synchronize()
                frames.append(hdr.cpu().numpy().copy())
        fields = {n: sc.get(n) for n in FIELDS}
        if precision == "checked":
            assert pkg.check_guards() == 0
        sc.close()
        if precision == "checked":
            assert pkg.check_guards() == 0
        runs[precision] = (fields, frames, cycles)
    got, want = runs["checked"], runs["f32"]
    assert got[2] == want[2]
    for n in FIELDS:
        _bits_equal(f"{dims}/{n}", got[0][n], want[0][n])
    for j, (g, w) in enumerate(zip(got[1], want[1])):
        _bits_equal(f"{dims}/frame{j}", g, w)


def test_batch_keeps_guards_and_bits(pkg, abi):
    """Three scenes of three shapes in one FireBatch (batched stage launches,
    one persistent multigrid launch), four sub-steps with a render on the
    last: no guard changes, and each scene equals the default build's."""
    sizes = [(24, 20, 16), (33, 17, 21), (40, 24, 28)]
    runs = {}
    for precision in ("checked", "f32"):
        pairs = [_config_scene(pkg, abi, d, k, precision) for k, d in enumerate(sizes)]
        scenes = [p[0] for p in pairs]
        batch = pkg.Batch(scenes)
        for i in range(4):
            s = [abi.FireSettings(width=48, height=32, dt=1.0 / 60.0, reset=1 if i == 0 else 0) for _ in scenes]
            batch.run(s, render=[i == 3] * len(scenes))
        batch.synchronize()
        out = [({n: sc.get(n) for n in FIELDS}, hdr.cpu().numpy().copy()) for sc, hdr in pairs]
        if precision == "checked":
            assert pkg.check_guards() == 0
        batch.close()
        for sc in scenes:
            sc.close()
        if precision == "checked":
            assert pkg.check_guards() == 0
        runs[precision] = out
    for k, ((gf, gh), (wf, wh)) in enumerate(zip(runs["checked"], runs["f32"])):
        for n in FIELDS:
            _bits_equal(f"{sizes[k]}/{n}", gf[n], wf[n])
        _bits_equal(f"{sizes[k]}/hdr", gh, wh)


def test_batched_server_keeps_guards_and_bits(pkg, abi):
    """Four config-physics requests of two shapes served in batched rounds:
    every one completes with no guard changes, and each served heat field and
    frame equals the default build's."""
    sizes = [(24, 28, 20), (32, 32, 32)]
    runs = {}
    for precision in ("checked", "f32"):
        server = pkg.Server(budget_bytes=64 << 30, precision=precision)
        heats, hdrs, reqs = [], [], []
        for i in range(4):
            dims = sizes[i % 2]
            r = abi.FireServeRequest()
            r.id = i
            r.nx, r.ny, r.nz = dims
            r.frameW, r.frameH = 64, 48
            r.steps, r.renderEvery, r.arrivalSeconds = 4 + i, 3, 0.005 * i
            r.physics = abi.config_scene(*dims, dims[0] / 2, dims[2] / 2, 3.0 + 0.5 * i, 0.3, -0.2, 200 + i)
            r.physics.pressureTop = 1
            r.multigridCycles, r.multigridPre, r.multigridPost, r.pressureTolerance = 20, 2, 2, 1e-5
            r.settings = abi.FireSettings(width=64, height=48, dt=1.0 / 60.0)
            heat = np.zeros(dims[::-1], dtype=np.float32)
            hdr = np.zeros((48, 64, 4), dtype=np.float32)
            r.resultHeat, r.resultHdr = heat.ctypes.data, hdr.ctypes.data
            reqs.append(r)
            heats.append(heat)
            hdrs.append(hdr)
            server.submit(r)
        rep = server.run(60.0)
        assert rep["completed"] == 4
        if precision == "checked":
            assert pkg.check_guards() == 0
        server.close()
        if precision == "checked":
            assert pkg.check_guards() == 0
        runs[precision] = (heats, hdrs)
    for i in range(4):
        _bits_equal(f"request {i} heat", runs["checked"][0][i], runs["f32"][0][i])
        _bits_equal(f"request {i} hdr", runs["checked"][1][i], runs["f32"][1][i])
        assert runs["f32"][0][i].sum() > 0.0


@pytest.mark.parametrize("dims", [(8, 8, 8), (17, 9, 5)])
def test_tiny_grids_keep_guards_and_follow_the_oracle(pkg, abi, oracle_mod, dims):
    """Grids smaller than one resident-SOR brick along every axis (every brick
    partial, light grid at its minimum size): four frames of the reference
    physics, rendered.  The checked build changes no guard byte; only then
    does the default build run them, equal to the checked build bit for bit.
    Against the CPU oracle the fields are compared in the TINY_GRID class:
    on so few cells the reaction's sin-hash noise, which the oracle cannot
    round as CUDA's sinf does, moves most burning cells (ash at 8^3: 3e-2
    relative L2 after four frames, 48 % of cells beyond 1e-5 of the field's
    scale).  The statistics are printed (pytest -s)."""
    import tolerances as T
    from conftest import STATE_FIELDS

    fields = STATE_FIELDS[:10] + ["u", "v", "w"]
    runs = {}
    for precision in ("checked", "f32"):
        sim = pkg.FireSim(48, 32, *dims, precision=precision)
        frames = []
        for f in range(4):
            s = abi.validation_settings(f, scene=0, width=48, height=32)
            s.reset = 1 if f == 0 else 0
            frames.append(sim.step_and_render(s)[0])
        sim.synchronize()
        runs[precision] = ({n: sim.get(n) for n in fields}, frames)
        if precision == "checked":
            assert pkg.check_guards() == 0
        sim.close()
        if precision == "checked":
            assert pkg.check_guards() == 0
    o = oracle_mod.OracleFire(abi, 48, 32, *dims)
    for f in range(4):
        s = abi.validation_settings(f, scene=0, width=48, height=32)
        s.reset = 1 if f == 0 else 0
        o.step(s, mode=2)
    (got, got_frames), (want, want_frames) = runs["checked"], runs["f32"]
    for n in fields:
        _bits_equal(f"{dims}/{n}", got[n], want[n])
    for j, (g, w) in enumerate(zip(got_frames, want_frames)):
        _bits_equal(f"{dims}/frame{j}", g, w)
    ref = {n: o.get(n) for n in fields}
    print(f"{dims} vs oracle (rel L2):", ", ".join(f"{n} {T.field_stats(want[n], ref[n])['rel_l2']:.1e}" for n in fields))
    for n in fields:
        T.check_field(f"{dims}/{n} vs oracle", want[n], ref[n], T.TINY_GRID)
    assert want["heat"].sum() > 0.0
