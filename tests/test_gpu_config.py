"""The config physics (FirePhysicsParams.mode 1) on the GPU against its CPU
oracle (oracle/config_oracle.cpp).

The config kernels are compiled without FMA contraction and the oracle
evaluates the same expressions in the same order in IEEE float, so every
simulation stage and whole trajectories are compared as bits.  The render
(transmittance and raymarch) uses expf, so it is compared within a stated
tolerance.  Precision: the FP32 and BF16-storage builds against the FP64
oracle, with the errors reported and bounded.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def product(pkg):
    return pkg


SIM_STAGES = ["advect_velocity", "advect_react", "force", "divergence", "pressure_sor", "subtract", "wall_boundary"]
STAGE_FIELDS = {
    "advect_velocity": ["u", "v", "w"], "advect_react": ["heat", "fuel", "soot"], "force": ["u", "v", "w"],
    "divergence": ["divergence", "pressure"], "pressure_sor": ["pressure"], "subtract": ["u", "v", "w"],
    "wall_boundary": ["u", "v", "w"],
}
STATE = ["heat", "fuel", "soot", "u", "v", "w", "pressure"]
# Render tolerance: expf differs between the device and the host C library by
# about an ulp, which the integrals carry as relative noise of ~1e-7 per sample.
RENDER_REL_L2 = 2e-6
RENDER_MAX_ABS = 2e-5


def _physics(abi, dims):
    """A C2-like scene with every term on: two emitters (one against a wall),
    confinement, curl noise of a short period, wind on x and z."""
    nx, ny, nz = dims
    p = abi.default_physics(*dims)
    p.mode = 1
    p.buoyancyHeat, p.buoyancySoot, p.vorticityEps = 1.0, 0.1, 0.3
    p.windX, p.windZ = 0.5, -0.3
    p.noiseAmplitude, p.noisePeriod, p.noiseSeed = 0.4, 7.0, 7
    p.emitterCount = 2
    p.emitters[0] = abi.FireEmitterDisk(centerX=nx / 2, centerY=2.0, centerZ=nz / 2, radius=min(nx, nz) / 5, fuel=1.0,
                                        heat=1.0, upVelocity=2.0, jitterScale=0.2, seed=1)
    p.emitters[1] = abi.FireEmitterDisk(centerX=0.0, centerY=1.0, centerZ=3.0, radius=3.0, fuel=0.6, heat=0.8,
                                        upVelocity=1.5, jitterScale=0.4, seed=3)
    p.primarySamples, p.lightSamples = 48, 24
    p.lightX, p.lightY, p.lightZ = nx * 0.3, ny * 1.5, nz * 0.6
    return p


def _pair(product, abi, oracle_mod, dims, frame=(40, 32), sor=(30, 1.8)):
    sim = product.FireSim(frame[0], frame[1], *dims)
    sim.set_physics(_physics(abi, dims))
    sim.set_pressure_solver(*sor)
    sim.reset()
    o = oracle_mod.ConfigOracle(abi, frame[0], frame[1], *dims)
    o.set_physics(_physics(abi, dims))
    o.set_pressure_solver(*sor)
    return sim, o


def _random_state(dims, seed):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    f = np.float32
    return {
        "heat": rng.uniform(0, 2, (nz, ny, nx)).astype(f), "fuel": rng.uniform(0, 1, (nz, ny, nx)).astype(f),
        "soot": rng.uniform(0, 0.3, (nz, ny, nx)).astype(f),
        "u": (0.7 * rng.standard_normal((nz, ny, nx + 1))).astype(f),
        "v": (0.7 * rng.standard_normal((nz, ny + 1, nx))).astype(f),
        "w": (0.7 * rng.standard_normal((nz + 1, ny, nx))).astype(f),
        "pressure": rng.standard_normal((nz, ny, nx)).astype(f),
        "divergence": (0.3 * rng.standard_normal((nz, ny, nx))).astype(f),
    }


def _bits_equal(name, got, want):
    g, w = got.view(np.uint32), want.view(np.uint32)
    bad = int(np.count_nonzero(g != w))
    if bad:
        d = np.abs(got.astype(np.float64) - want.astype(np.float64))
        raise AssertionError(f"{name}: {bad}/{got.size} values differ, max |diff| {d.max():.3e}")


@pytest.mark.parametrize("dims", [(24, 20, 18), (33, 17, 21), (16, 16, 16)])
def test_config_stages_equal_the_oracle_bitwise(dims, product, abi, oracle_mod):
    """Each simulation stage from the same random state (velocities of ~0.7
    cells/step, so backtraces cross cells and walls) gives the oracle's bits."""
    s = abi.FireSettings()
    for k, stage in enumerate(SIM_STAGES):
        sim, o = _pair(product, abi, oracle_mod, dims)
        for n, a in _random_state(dims, 100 + k).items():
            sim.set(n, a)
            o.set(n, a)
        sim.set("oxygen", np.zeros(dims[::-1], np.float32))
        sim.stages(stage, stage, s, 0.0)
        o.stages(stage, stage)
        for n in STAGE_FIELDS[stage]:
            _bits_equal(f"{dims}/{stage}/{n}", sim.get(n), o.get(n))
        sim.close()


def test_config_trajectory_equals_the_oracle_bitwise(product, abi, oracle_mod):
    """25 whole steps from an empty scene (emitters, burn, confinement, noise,
    wind, projection): every field of the state as bits."""
    dims = (40, 36, 44)
    sim, o = _pair(product, abi, oracle_mod, dims)
    s = abi.FireSettings()
    for _ in range(25):
        sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        o.step()
    for n in STATE:
        _bits_equal(f"step25/{n}", sim.get(n), o.get(n))
    assert sim.get("heat").sum() > 1.0 and sim.get("soot").sum() > 0.0
    sim.close()


def test_config_render_matches_the_oracle(product, abi, oracle_mod):
    """Transmittance volume and HDR frame after 20 steps, within the expf tolerance."""
    dims = (32, 40, 28)
    sim, o = _pair(product, abi, oracle_mod, dims, frame=(64, 48))
    s = abi.FireSettings()
    for _ in range(20):
        sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        o.step()
    sim.stages("light_build", "render", s, 0.0)
    o.stages("light_build", "render")
    for n in ("config_transmittance", "hdr"):
        got, want = sim.get(n).astype(np.float64), o.get(n).astype(np.float64)
        rel = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert rel <= RENDER_REL_L2 and np.abs(got - want).max() <= RENDER_MAX_ABS, (n, rel, np.abs(got - want).max())
    tr = sim.get("config_transmittance")
    assert 0.0 < tr.min() < 1.0 and tr.max() <= 1.0
    hdr = sim.get("hdr")
    assert hdr[..., 3].max() > 0.05 and np.isfinite(hdr).all()
    sim.close()


@pytest.mark.parametrize("precision,bound", [("f32", 1e-4), ("bf16", 5e-2)])
def test_config_precision_against_the_fp64_oracle(precision, bound, product, abi, oracle_mod):
    """30 steps at 48^3 (the C3 pattern at a size the FP64 oracle finishes in
    seconds): relative L2 error of each field against the FP64 oracle."""
    dims = (48, 48, 48)
    sim = product.FireSim(32, 24, *dims, precision=precision)
    p = _physics(abi, dims)
    sim.set_physics(p)
    sim.set_pressure_solver(60, 1.85)
    sim.reset()
    o = oracle_mod.ConfigOracle(abi, 32, 24, *dims, precision="f64")
    o.set_physics(p)
    o.set_pressure_solver(60, 1.85)
    s = abi.FireSettings()
    for _ in range(30):
        sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        o.step()
    errors = {}
    for n in ("heat", "fuel", "soot", "u", "v", "w"):
        got, want = sim.get(n).astype(np.float64), o.get64(n)
        errors[n] = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    print(precision, errors)
    assert max(errors.values()) <= bound, errors
    sim.close()


def test_config_scenes_and_batches_equal_the_singleton(product, abi):
    """Two FireScene handles in config physics stepped by fireBatchStep give the
    singleton's bits."""
    dims = (32, 24, 28)
    p = _physics(abi, dims)
    s = abi.FireSettings()
    s.reset = 0
    sim = product.FireSim(32, 24, *dims)
    sim.set_physics(p)
    sim.set_pressure_solver(30, 1.8)
    sim.reset()
    for _ in range(8):
        sim.step(s)
    want = {n: sim.get(n) for n in ("heat", "soot", "u", "v", "w")}
    sim.close()
    scenes = [product.firesim.Scene(32, 24, *dims) for _ in range(2)]
    for sc in scenes:
        sc.set_physics(p)
        sc.set_pressure_solver(30, 1.8)
        sc.step(abi.FireSettings(reset=1))  # the reset frame zeroes the config fields, then steps
    for _ in range(7):
        product.firesim.batch_step(scenes, [s, s])
    for sc in scenes:
        for n, a in want.items():
            _bits_equal(f"scene/{n}", sc.get(n), a)
        sc.close()


def test_config_physics_validation(product, abi):
    sim = product.FireSim(32, 24, 16, 16, 16)
    bad = []
    for field, value in (("mode", 2), ("primarySamples", 0), ("emitterCount", 5), ("dt", float("nan")),
                         ("noisePeriod", 0.0), ("fovYDegrees", 180.0)):
        p = abi.default_physics(16, 16, 16)
        p.mode = 1
        setattr(p, field, value)
        with pytest.raises(product.firesim.FireSimError, match="physic|emitter"):
            sim.set_physics(p)
        bad.append(field)
    p = abi.default_physics(16, 16, 16)
    p.mode = 1
    sim.set_physics(p)
    assert sim.physics().mode == 1
    sim.close()


def test_config_gated_solve_on_both_paths(product, abi):
    """The C3 solver policy (max |r| <= tolerance or the iteration cap) in config
    physics, on the resident path and the colour-split path, gives one result."""
    dims = (64, 64, 64)
    p = _physics(abi, dims)
    s = abi.FireSettings()
    out = []
    for path in (2, 1):
        sim = product.FireSim(32, 24, *dims)
        sim.set_physics(p)
        sim.set_pressure_solver(120, 1.85)
        sim.set_pressure_tolerance(1e-3, 10)
        sim.set_pressure_path(path)
        sim.reset()
        for _ in range(10):
            sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        assert sim.pressure_path_used() == path
        stats = sim.pressure_stats()
        assert stats[0] <= 120 and (stats[1] <= 1e-3 or stats[0] == 120)
        out.append((stats, {n: sim.get(n) for n in ("pressure", "u", "v", "w")}))
        sim.close()
    assert out[0][0][0] == out[1][0][0]
    for n in out[0][1]:
        _bits_equal(f"gated/{n}", out[0][1][n], out[1][1][n])


@pytest.mark.parametrize("dims,cycles,tol", [((32, 32, 32), 12, 1e-5), ((64, 48, 40), 12, 1e-5), ((33, 17, 21), 5, 0.0),
                                             ((128, 128, 128), 10, 1e-5), ((125, 4, 99), 3, 0.0), ((20, 36, 44), 6, 0.0),
                                             ((41, 37, 35), 2, 0.0)])
def test_multigrid_equals_the_oracle_bitwise(dims, cycles, tol, product, abi, oracle_mod):
    """The multigrid solve (Dirichlet top) from a random right-hand side: the
    same pressure bits and the same number of V-cycles as the oracle, gated
    and fixed.  The shapes cover the solve's tail (the coarse end of the
    hierarchy, one CTA) in its three modes: all in shared memory (from 32^3
    down at 32^3, with a one-warp 2^3 coarsest level; 64x48x40,
    semi-coarsened to 2x3x5; 33x17x21, which cannot coarsen, so the tail is
    level 0; 125x2x99 below 125x4x99); the tail level's rhs in global memory
    (from 32^3 down at 128^3); and all in global memory (41x37x35, which
    cannot coarsen and is too large for shared memory)."""
    p = abi.default_physics(*dims)
    p.mode, p.pressureTop = 1, 1
    d = (0.3 * np.random.default_rng(4).standard_normal(dims[::-1])).astype(np.float32)
    sim = product.FireSim(32, 16, *dims)
    sim.set_physics(p)
    sim.set_pressure_multigrid(cycles, 2, 2)
    sim.set_pressure_tolerance(tol, 1)
    sim.set("divergence", d)
    sim.set("pressure", np.zeros_like(d))
    sim.stages("pressure_sor", "pressure_sor", abi.FireSettings(), 0.0)
    assert sim.pressure_path_used() == 3
    o = oracle_mod.ConfigOracle(abi, 32, 16, *dims)
    o.set_physics(p)
    o.set_multigrid(cycles, 2, 2, tol)
    o.set("divergence", d)
    o.set("pressure", np.zeros_like(d))
    o.stages("pressure_sor", "pressure_sor")
    _bits_equal(f"mg{dims}", sim.get("pressure"), o.get("pressure"))
    if tol > 0:
        stats, (oc, om) = sim.pressure_stats(), o.multigrid_stats()
        assert stats[0] == oc and stats[1] == om and om <= tol, (stats, oc, om)
    sim.close()


def test_config_dirichlet_trajectory_meets_the_divergence_bound(product, abi, oracle_mod):
    """Config physics with the Dirichlet top and the multigrid solve (max |r| <=
    1e-5): 15 steps equal the oracle bit for bit, and after every projection
    the divergence of the velocity (every cell, top faces included) is below
    1e-4."""
    dims = (48, 40, 44)
    p = _physics(abi, dims)
    p.pressureTop = 1
    sim = product.FireSim(32, 16, *dims)
    sim.set_physics(p)
    sim.set_pressure_multigrid(30, 2, 2)
    sim.set_pressure_tolerance(1e-5, 1)
    sim.reset()
    o = oracle_mod.ConfigOracle(abi, 32, 16, *dims)
    o.set_physics(p)
    o.set_multigrid(30, 2, 2, 1e-5)
    s = abi.FireSettings()
    for step in range(15):
        sim.stages("advect_velocity", "wall_boundary", s, 0.0)
        o.step()
        u, v, w = sim.get("u"), sim.get("v"), sim.get("w")
        div = (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:] - w[:-1])
        assert np.abs(div).max() <= 1e-4, (step, np.abs(div).max())
    for n in STATE:
        _bits_equal(f"dirichlet/{n}", sim.get(n), o.get(n))
    sim.close()


def test_solver_and_top_must_match(product, abi):
    dims = (16, 16, 16)
    sim = product.FireSim(32, 16, *dims)
    s = abi.FireSettings()
    p = abi.default_physics(*dims)
    p.mode, p.pressureTop = 1, 1
    sim.set_physics(p)
    with pytest.raises(product.firesim.FireSimError, match="needs the multigrid"):
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
    p.pressureTop = 0
    sim.set_physics(p)
    sim.set_pressure_multigrid(4)
    with pytest.raises(product.firesim.FireSimError, match="Dirichlet top"):
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
    with pytest.raises(product.firesim.FireSimError, match="multigrid"):
        sim.set_pressure_multigrid(4, 0, 2)
    sim.close()
