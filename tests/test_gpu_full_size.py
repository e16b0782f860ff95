"""The single-scene config-physics workloads at their own sizes and lengths
(needs a GPU; abi.config_workload states them):

  c1: 64^3, 100 steps, then one 256^2 frame;
  c2: 128^3, 200 steps, a 512^2 frame every 10 steps;
  c3: 256^3, 100 steps, SOR until max |r| <= 1e-5 or 120 iterations, in BF16
      storage (and FP16 and FP32 beside it) against the FP64 oracle.

The config physics has no counterpart in native-firesim, so its oracle is the
CPU restatement oracle/config_oracle.cpp (self-oracled).  c1 and c2 are
compared with the float oracle bit for bit on every field of the state, and
their frames within the render tolerance (expf differs by an ulp between the
device and the host C library).  c3 compares each storage build with the
FP64 oracle by relative L2 per field, and reports the post-projection
divergence both of the stored velocity and of the float velocity before it
is rounded to storage.  The measured values are printed (pytest -s).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ("heat", "fuel", "soot", "u", "v", "w", "pressure")
RENDER_REL_L2 = 2e-6
RENDER_MAX_REL = 2e-5


def _bits_equal(name, got, want):
    g, w = np.ascontiguousarray(got).view(np.uint32), np.ascontiguousarray(want).view(np.uint32)
    bad = int(np.count_nonzero(g != w))
    assert bad == 0, f"{name}: {bad}/{g.size} values differ, max |diff| {np.abs(got.astype(np.float64) - want).max():.3e}"


def _frame_close(name, got, want):
    got, want = got.astype(np.float64), want.astype(np.float64)
    rel = float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))
    mx = float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-30))
    assert rel <= RENDER_REL_L2 and mx <= RENDER_MAX_REL, (name, rel, mx)
    return rel, mx


def _gpu_scene(pkg, w, precision="f32"):
    fw, fh = w["frame"]
    sim = pkg.FireSim(fw, fh, *w["grid"], precision=precision)
    sim.set_physics(w["physics"])
    sim.set_pressure_solver(*w["sor"])
    if w["tolerance"] > 0:
        sim.set_pressure_tolerance(w["tolerance"], w["check_every"])
    sim.reset()
    return sim


def _oracle(oracle_mod, abi, w, precision="f32"):
    fw, fh = w["frame"]
    o = oracle_mod.ConfigOracle(abi, fw, fh, *w["grid"], precision=precision)
    o.set_physics(w["physics"])
    o.set_pressure_solver(*w["sor"])
    return o


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_config_workload_equals_the_oracle_at_full_size(name, pkg, abi, oracle_mod):
    w = abi.config_workload(name)
    assert w["tolerance"] == 0.0
    sim = _gpu_scene(pkg, w)
    o = _oracle(oracle_mod, abi, w)
    s = abi.FireSettings()
    checks = {w["steps"]} | ({50, 100, 150} if name == "c2" else set())
    frames = []
    for step in range(1, w["steps"] + 1):
        render = step % w["render_every"] == 0
        sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        o.step(render=render)
        if render:
            sim.stages("light_build", "render", s, 0.0)
            frames.append(_frame_close(f"{name}/frame{step}", sim.get("hdr"), o.get("hdr")))
        if step in checks:
            for n in STATE:
                _bits_equal(f"{name}/step{step}/{n}", sim.get(n), o.get(n))
    heat = sim.get("heat")
    assert heat.max() > 0.5 and np.isfinite(heat).all()
    print(f"{name}: {w['steps']} steps bit-identical on {len(checks)} checks; {len(frames)} frames, "
          f"worst rel-L2 {max(f[0] for f in frames):.2e}, worst max-rel {max(f[1] for f in frames):.2e}")
    sim.close()


def _divergence(u, v, w):
    u, v, w = (a.astype(np.float64) for a in (u, v, w))
    return (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:] - w[:-1])


def _projected_f32(u, v, w, p):
    """The SOR path's subtraction and walls in float (subtractWall): the
    velocity the projection computes before it is rounded to storage."""
    u, v, w, p = (a.astype(np.float32).copy() for a in (u, v, w, p))
    u[:, :, 1:-1] -= p[:, :, 1:] - p[:, :, :-1]
    v[:, 1:-1, :] -= p[:, 1:, :] - p[:, :-1, :]
    w[1:-1] -= p[1:] - p[:-1]
    u[:, :, 0] = u[:, :, -1] = 0.0
    v[:, 0, :] = 0.0
    w[0] = w[-1] = 0.0
    return u, v, w


@pytest.mark.slow
def test_c3_storage_builds_against_the_fp64_oracle(pkg, abi, oracle_mod):
    """c3 at 256^3 after 100 steps: each storage build's relative L2 error per
    field against the FP64 oracle of the same seeds.  Measured on the B200:
    FP32 <= 6.5e-6, FP16 <= 7.9e-3, BF16 <= 7.6e-2 (the storage rounding of
    every transported field, 2^-12 and 2^-9 relative per step, accumulates
    over the 100 steps; neither 16-bit format meets 1e-3).  Bounds: FP32 1e-4,
    FP16 1.5e-2, BF16 0.12."""
    w = abi.config_workload("c3")
    steps = w["steps"]
    o = _oracle(oracle_mod, abi, w, precision="f64")
    oracle_mod.OracleFire.set_threads(os.cpu_count() or 1)
    for _ in range(steps):
        o.step()
    want = {n: o.get64(n) for n in ("heat", "fuel", "soot", "u", "v", "w")}
    s = abi.FireSettings()
    bounds = {"f32": 1e-4, "f16": 1.5e-2, "bf16": 0.12}
    report = {}
    for precision, bound in bounds.items():
        sim = _gpu_scene(pkg, w, precision)
        for _ in range(steps - 1):
            sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        sim.stages("advect_velocity", "pressure_sor", s, 0.0)
        pre = [sim.get(n) for n in ("u", "v", "w", "pressure")]
        div_f32 = float(np.abs(_divergence(*_projected_f32(*pre))).max())
        sim.stages("subtract", "wall_boundary", s, 0.0)
        div_stored = float(np.abs(_divergence(sim.get("u"), sim.get("v"), sim.get("w"))).max())
        errors = {n: float(np.linalg.norm(sim.get(n).astype(np.float64) - a) / np.linalg.norm(a)) for n, a in want.items()}
        iterations, max_r, _ = sim.pressure_stats()
        report[precision] = (errors, div_stored, div_f32, iterations, max_r)
        print(f"c3 {precision}: rel-L2 {errors}; |div u| stored {div_stored:.2e}, before rounding {div_f32:.2e}; "
              f"SOR {iterations} iterations, max|r| {max_r:.2e}")
        assert max(errors.values()) <= bound, (precision, errors)
        sim.close()
    assert report["f16"][0]["heat"] < report["bf16"][0]["heat"]
