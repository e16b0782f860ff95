"""FireBatch: scenes of the config physics stepped together, one launch per
stage over all of them and one persistent multigrid launch for every
scene's pressure solve (needs a GPU).

A batched scene runs the single-scene kernels' own per-element work, so its
state and frames must equal the same scene stepped alone, bit for bit, and
its multigrid must run the same number of cycles.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(24, 20, 16), (32, 32, 32), (40, 24, 28), (16, 48, 20), (33, 17, 21), (64, 48, 40)]
FIELDS = ("heat", "fuel", "soot", "u", "v", "w", "pressure")


def _physics(abi, dims, k):
    nx, ny, nz = dims
    p = abi.default_physics(*dims)
    p.mode, p.pressureTop = 1, 1
    p.buoyancyHeat, p.buoyancySoot, p.vorticityEps = 1.0, 0.1, 0.3 if k % 2 == 0 else 0.0
    p.windX, p.windZ = 0.4 - 0.1 * k, 0.2
    p.noiseAmplitude, p.noisePeriod, p.noiseSeed = (0.4, 7.0, 7 + k) if k % 3 != 1 else (0.0, 16.0, 1)
    p.emitterCount = 1
    p.emitters[0] = abi.FireEmitterDisk(centerX=nx / 2, centerY=2.0, centerZ=nz / 2, radius=max(2.0, min(nx, nz) / 5), fuel=1.0,
                                        heat=1.0, upVelocity=2.0, jitterScale=0.2, seed=100 + k)
    p.primarySamples, p.lightSamples = 32, 16
    p.lightX, p.lightY, p.lightZ = nx * 0.5, ny * 1.5, nz * 0.5
    return p


def _scene(pkg, abi, dims, k, frame=(48, 32)):
    import torch

    sc = pkg.Scene(frame[0], frame[1], *dims)
    sc.set_physics(_physics(abi, dims, k))
    sc.set_pressure_multigrid(20, 2, 2)
    sc.set_pressure_tolerance(1e-5, 1)
    hdr = torch.zeros((frame[1], frame[0], 4), dtype=torch.float32, device="cuda")
    sc.set_hdr_buffer(hdr.data_ptr(), frame[0] * 16, 0)
    return sc, hdr


def _bits_equal(name, got, want):
    g, w = np.ascontiguousarray(got).view(np.uint32), np.ascontiguousarray(want).view(np.uint32)
    bad = int(np.count_nonzero(g != w))
    assert bad == 0, f"{name}: {bad}/{g.size} values differ, max |diff| {np.abs(got.astype(np.float64) - want).max():.3e}"


def test_batch_equals_each_scene_alone(pkg, abi):
    """Six scenes of six shapes (odd, flat and ragged ones included), eight
    sub-steps with a render on the fourth and the eighth: every field, the
    HDR frames and the multigrid cycle counts equal each scene stepped alone."""
    steps, renders = 8, {3, 7}
    settings = abi.FireSettings(width=48, height=32, dt=1.0 / 60.0)
    alone = []
    for k, dims in enumerate(SIZES):
        sc, hdr = _scene(pkg, abi, dims, k)
        frames, cycles = [], []
        for i in range(steps):
            settings.reset = 1 if i == 0 else 0
            sc.step(settings, render=i in renders)
            cycles.append(sc.pressure_stats()[0])
            if i in renders:
                sc.synchronize()
                frames.append(hdr.cpu().numpy().copy())
        alone.append(({n: sc.get(n) for n in FIELDS}, frames, cycles))
        sc.close()

    pairs = [_scene(pkg, abi, dims, k) for k, dims in enumerate(SIZES)]
    scenes = [p[0] for p in pairs]
    batch = pkg.Batch(scenes)
    frames = [[] for _ in scenes]
    cycles = [[] for _ in scenes]
    for i in range(steps):
        s = []
        for _ in scenes:
            t = abi.FireSettings(width=48, height=32, dt=1.0 / 60.0)
            t.reset = 1 if i == 0 else 0
            s.append(t)
        batch.run(s, render=[i in renders] * len(scenes))
        batch.synchronize()
        for k, sc in enumerate(scenes):
            cycles[k].append(sc.pressure_stats()[0])
            if i in renders:
                frames[k].append(pairs[k][1].cpu().numpy().copy())
    assert batch.launch_count() > 0
    for k, sc in enumerate(scenes):
        want_fields, want_frames, want_cycles = alone[k]
        assert cycles[k] == want_cycles, (SIZES[k], cycles[k], want_cycles)
        for n in FIELDS:
            _bits_equal(f"{SIZES[k]}/{n}", sc.get(n), want_fields[n])
        for j, (g, w) in enumerate(zip(frames[k], want_frames)):
            _bits_equal(f"{SIZES[k]}/frame{j}", g, w)
        assert want_fields["heat"].sum() > 0.0
    batch.close()
    for sc in scenes:
        sc.close()


def test_batch_projection_meets_the_divergence_bound(pkg, abi):
    """After each batched sub-step every scene's velocity is divergence-free
    to 1e-4 (max over cells, top faces included)."""
    pairs = [_scene(pkg, abi, dims, k) for k, dims in enumerate(SIZES[:3])]
    scenes = [p[0] for p in pairs]
    batch = pkg.Batch(scenes)
    for i in range(12):
        s = [abi.FireSettings(width=48, height=32, dt=1.0 / 60.0, reset=1 if i == 0 else 0) for _ in scenes]
        batch.run(s)
        batch.synchronize()
        for sc in scenes:
            u, v, w = sc.get("u"), sc.get("v"), sc.get("w")
            div = (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:] - w[:-1])
            assert np.abs(div).max() <= 1e-4, (i, np.abs(div).max())
    batch.close()
    for sc in scenes:
        sc.close()


def test_batch_rejects_scenes_without_the_multigrid_projection(pkg, abi):
    sc = pkg.Scene(32, 16, 16, 16, 16)
    p = abi.default_physics(16, 16, 16)
    p.mode = 1
    sc.set_physics(p)
    sc.set_pressure_solver(20, 1.8)
    with pytest.raises(pkg.FireSimError, match="multigrid"):
        pkg.Batch([sc])
    sc.close()
