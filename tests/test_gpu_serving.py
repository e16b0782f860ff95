"""Independent scenes, batched steps and the serving loop (needs a GPU).

Scenes share nothing on the device, so a scene's result must be the same bits
whether it runs through the singleton ABI, through its own FireScene handle,
side by side with others in fireBatchStep, or admitted by the server into a
mix of requests that arrive over time.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(24, 28, 20), (32, 32, 32), (40, 24, 36)]


def _settings(abi, f, scene=0, w=64, h=48):
    s = abi.validation_settings(f, scene=scene, width=w, height=h)
    s.reset = 1 if f == 0 else 0
    return s


def _alone(pkg, abi, dims, steps, render_every, scene=0, settings=None):
    import torch
    nx, ny, nz = dims
    sc = pkg.Scene(64, 48, nx, ny, nz)
    hdr = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
    sc.set_hdr_buffer(hdr.data_ptr(), 64 * 16, 0)
    for f in range(steps):
        s = settings(f) if settings else _settings(abi, f, scene)
        sc.step(s, render=render_every > 0 and f % render_every == render_every - 1)
    sc.synchronize()
    out = {n: sc.get(n) for n in ("heat", "fuel", "soot", "u", "v", "w", "pressure")}
    torch.cuda.synchronize()
    out["hdr"] = hdr.cpu().numpy()
    sc.close()
    return out


def test_scene_handle_equals_singleton(pkg, abi):
    """A FireScene steps exactly like the reference-style singleton."""
    nx, ny, nz = SIZES[1]
    sim = pkg.FireSim(64, 48, nx, ny, nz)
    for f in range(6):
        sim.step(_settings(abi, f))
    sim.synchronize()
    want = {n: sim.get(n) for n in ("heat", "fuel", "soot", "u", "v", "w", "pressure")}
    sim.close()
    got = _alone(pkg, abi, SIZES[1], 6, 0)
    for n, a in want.items():
        np.testing.assert_array_equal(got[n].view(np.uint32), a.view(np.uint32), err_msg=n)


def test_batch_step_equals_alone(pkg, abi):
    """Three scenes of different sizes and scenes, stepped together with fireBatchStep
    (a render every 3rd step), equal each scene stepped alone."""
    import torch
    scenes = [pkg.Scene(64, 48, *d) for d in SIZES]
    hdrs = [torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda") for _ in SIZES]
    for sc, hdr in zip(scenes, hdrs):
        sc.set_hdr_buffer(hdr.data_ptr(), 64 * 16, 0)
    for f in range(7):
        pkg.batch_step(scenes, [_settings(abi, f, scene=i) for i in range(3)], render=[f % 3 == 2] * 3)
    for i, (sc, hdr) in enumerate(zip(scenes, hdrs)):
        sc.synchronize()
        alone = _alone(pkg, abi, SIZES[i], 7, 3, scene=i)
        for n in ("heat", "fuel", "soot", "u", "v", "w", "pressure"):
            np.testing.assert_array_equal(sc.get(n).view(np.uint32), alone[n].view(np.uint32), err_msg=f"scene {i} {n}")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(hdr.cpu().numpy().view(np.uint32), alone["hdr"].view(np.uint32), err_msg=f"scene {i} hdr")
        sc.close()


def _request(abi, rid, dims, steps, arrival, scene, render_every=4):
    r = abi.FireServeRequest()
    r.id = rid
    r.nx, r.ny, r.nz = dims
    r.frameW, r.frameH = 64, 48
    r.steps = steps
    r.renderEvery = render_every
    r.arrivalSeconds = arrival
    r.settings = _settings(abi, 1, scene=scene)
    return r


def test_server_results_equal_alone(pkg, abi):
    """Six requests of three sizes arrive over 60 ms; every one completes, and each
    request's final heat field and last frame equal the same request run alone."""
    server = pkg.Server(budget_bytes=64 << 30)
    reqs, heats, hdrs = [], [], []
    for i in range(6):
        dims = SIZES[i % 3]
        r = _request(abi, i, dims, steps=6 + 2 * i, arrival=0.01 * i, scene=i % 3)
        heat = np.zeros(dims[::-1], dtype=np.float32)
        hdr = np.zeros((48, 64, 4), dtype=np.float32)
        r.resultHeat, r.resultHdr = heat.ctypes.data, hdr.ctypes.data
        reqs.append(r)
        heats.append(heat)
        hdrs.append(hdr)
        server.submit(r)
    rep = server.run(60.0)
    server.close()
    assert rep["submitted"] == 6 and rep["completed"] == 6
    assert rep["voxelSteps"] == sum((6 + 2 * i) * np.prod(SIZES[i % 3]) for i in range(6))
    assert 0 < rep["stepMsP50"] <= rep["stepMsP99"] <= rep["stepMsMax"]
    for i, r in enumerate(reqs):
        base = r.settings

        def per_step(f, base=base):
            s = abi.FireSettings.from_buffer_copy(base)
            s.reset = 1 if f == 0 else 0
            return s

        alone = _alone(pkg, abi, SIZES[i % 3], r.steps, 4, settings=per_step)
        np.testing.assert_array_equal(heats[i].view(np.uint32), alone["heat"].view(np.uint32), err_msg=f"request {i} heat")
        np.testing.assert_array_equal(hdrs[i].view(np.uint32), alone["hdr"].view(np.uint32), err_msg=f"request {i} hdr")


def test_server_respects_budget(pkg, abi):
    """With room for about two scenes at a time, the server never holds more than
    its budget and still completes every request, later ones after a queue wait."""
    probe = pkg.Scene(64, 48, *SIZES[1])
    per_scene = probe.device_bytes() + 64 * 48 * 16
    probe.close()
    budget = int(2.5 * per_scene)
    server = pkg.Server(budget_bytes=budget)
    for i in range(5):
        server.submit(_request(abi, i, SIZES[1], steps=8, arrival=0.0, scene=0))
    rep = server.run(60.0)
    server.close()
    assert rep["completed"] == 5
    assert rep["admittedPeak"] <= 2
    assert rep["deviceBytesPeak"] <= budget
    assert rep["queueMsP99"] > 0.0


def test_server_pool_and_voxel_limit(pkg, abi):
    """With room for one active scene at a time (by cells), eight requests of two
    shapes run one after another; finished scenes are reused from the pool, and
    every request's result equals the same request run alone."""
    server = pkg.Server(budget_bytes=64 << 30)
    server.set_limits(int(np.prod(SIZES[2])))
    reqs, heats = [], []
    for i in range(8):
        dims = SIZES[i % 2]
        r = _request(abi, i, dims, steps=5 + i, arrival=0.0, scene=i % 3)
        heat = np.zeros(dims[::-1], dtype=np.float32)
        r.resultHeat = heat.ctypes.data
        reqs.append(r)
        heats.append(heat)
        server.submit(r)
    rep = server.run(60.0)
    assert rep["completed"] == 8 and rep["admittedPeak"] == 1
    # A second run on the same server starts from the pool.
    again = _request(abi, 8, SIZES[0], steps=5, arrival=0.0, scene=0)
    heat_again = np.zeros(SIZES[0][::-1], dtype=np.float32)
    again.resultHeat = heat_again.ctypes.data
    server.submit(again)
    assert server.run(60.0)["completed"] == 1
    server.close()
    for i, r in enumerate(reqs + [again]):
        base = r.settings

        def per_step(f, base=base):
            s = abi.FireSettings.from_buffer_copy(base)
            s.reset = 1 if f == 0 else 0
            return s

        alone = _alone(pkg, abi, (r.nx, r.ny, r.nz), r.steps, 4, settings=per_step)
        got = heats[i] if i < 8 else heat_again
        np.testing.assert_array_equal(got.view(np.uint32), alone["heat"].view(np.uint32), err_msg=f"request {i}")


def test_server_config_physics_equals_alone(pkg, abi):
    """Requests that carry config physics (one disk emitter each, their own
    seeds and wind) mixed with reference-physics requests: each served result
    equals the same scene stepped alone, and the pooled scenes switch physics
    between requests."""
    import torch
    server = pkg.Server(budget_bytes=64 << 30)
    reqs, heats = [], []
    for i in range(5):
        dims = SIZES[i % 2]
        r = _request(abi, i, dims, steps=8, arrival=0.01 * i, scene=0)
        if i % 2 == 0:
            r.physics = abi.config_scene(*dims, dims[0] / 2 + i, dims[2] / 2, 4.0 + i, 0.3, -0.2, 100 + i)
            r.settings = abi.FireSettings(width=64, height=48, dt=1.0 / 60.0)
        heat = np.zeros(dims[::-1], dtype=np.float32)
        r.resultHeat = heat.ctypes.data
        reqs.append(r)
        heats.append(heat)
        server.submit(r)
    rep = server.run(60.0)
    server.close()
    assert rep["completed"] == 5
    for i, r in enumerate(reqs):
        dims = SIZES[i % 2]
        sc = pkg.Scene(64, 48, *dims)
        hdr = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
        sc.set_hdr_buffer(hdr.data_ptr(), 64 * 16, 0)
        if r.physics.mode == 1:
            sc.set_physics(r.physics)
        for f in range(r.steps):
            s = abi.FireSettings.from_buffer_copy(r.settings)
            s.reset = 1 if f == 0 else 0
            sc.step(s, render=f % 4 == 3)
        alone = sc.get("heat")
        sc.close()
        np.testing.assert_array_equal(heats[i].view(np.uint32), alone.view(np.uint32), err_msg=f"request {i}")
        assert heats[i].sum() > 0.0


def test_server_rejects_invalid_physics(pkg, abi):
    server = pkg.Server(budget_bytes=1 << 30)
    r = _request(abi, 0, SIZES[0], steps=2, arrival=0.0, scene=0)
    r.physics = abi.config_scene(*SIZES[0], 10.0, 10.0, 3.0, 0.0, 0.0, 1)
    r.physics.lightSamples = 0
    with pytest.raises(pkg.firesim.FireSimError, match="sample counts"):
        server.submit(r)
    server.close()


@pytest.mark.parametrize("round_ms", [0.0, 0.3])
def test_batched_server_equals_alone(pkg, abi, round_ms):
    """Requests of the config physics with the multigrid projection are served
    as one batch per round (every admitted scene advanced by one launch per
    stage); with room for about two scenes by cells, eight requests of three
    shapes arrive over 40 ms, queue for free scenes and complete, and each
    served heat field and last frame equal the same scene stepped alone.
    With a round-time target (0.3 ms: tighter than most rounds) admission
    waits for the predicted round time, which changes the mix and not the
    results."""
    import torch
    server = pkg.Server(budget_bytes=64 << 30)
    server.set_limits(int(np.prod(SIZES[1]) + np.prod(SIZES[2])))
    if round_ms > 0:
        server.set_latency_target(round_ms)
    reqs, heats, hdrs = [], [], []
    for i in range(8):
        dims = SIZES[i % 3]
        r = _request(abi, i, dims, steps=5 + i, arrival=0.005 * i, scene=0, render_every=3)
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
    server.close()
    assert rep["completed"] == 8 and 1 <= rep["admittedPeak"] <= 3
    assert rep["voxelSteps"] == sum((5 + i) * np.prod(SIZES[i % 3]) for i in range(8))
    assert 0 < rep["stepMsP50"] <= rep["stepMsP99"] <= rep["stepMsMax"]
    for i, r in enumerate(reqs):
        dims = SIZES[i % 3]
        sc = pkg.Scene(64, 48, *dims)
        hdr = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
        sc.set_hdr_buffer(hdr.data_ptr(), 64 * 16, 0)
        sc.set_physics(r.physics)
        sc.set_pressure_multigrid(20, 2, 2)
        sc.set_pressure_tolerance(1e-5, 1)
        for f in range(r.steps):
            s = abi.FireSettings.from_buffer_copy(r.settings)
            s.reset = 1 if f == 0 else 0
            sc.step(s, render=f % 3 == 2)
        sc.synchronize()
        alone_heat = sc.get("heat")
        alone_hdr = hdr.cpu().numpy()
        sc.close()
        np.testing.assert_array_equal(heats[i].view(np.uint32), alone_heat.view(np.uint32), err_msg=f"request {i} heat")
        np.testing.assert_array_equal(hdrs[i].view(np.uint32), alone_hdr.view(np.uint32), err_msg=f"request {i} hdr")
        assert heats[i].sum() > 0.0
