"""The config physics (FirePhysicsParams.mode 1) without a GPU: the CPU oracle
against independent restatements of its pieces, and the host-side parameter
logic of the library.

The GPU tests (test_gpu_config.py) then hold the product to this oracle bit
for bit, so what is pinned here is pinned for the product too.
"""
from __future__ import annotations

import numpy as np
import pytest

M64 = (1 << 64) - 1


def splitmix64(z: int) -> int:
    """SplitMix64's output function (Steele, Lea and Flood, OOPSLA 2014), in Python integers."""
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def jitter(seed: int, step: int, cell: int) -> np.float32:
    k = ((seed << 32) ^ ((step * 0xD1B54A32D192ED03) & M64) ^ cell) & M64
    return np.float32(splitmix64(k) >> 40) * np.float32(1.0 / 16777216.0)


def disk_cells(nx, ny, nz, e):
    row = int(np.floor(e.centerY))
    z, x = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(nx, dtype=np.float32), indexing="ij")
    dx, dz = x - np.float32(e.centerX), z - np.float32(e.centerZ)
    inside = dx * dx + dz * dz <= np.float32(e.radius) * np.float32(e.radius)
    return row, inside


def _oracle(abi, oracle_mod, dims, physics, frame=(32, 24), precision="f32"):
    o = oracle_mod.ConfigOracle(abi, frame[0], frame[1], *dims, precision=precision)
    o.set_physics(physics)
    return o


def _physics(abi, dims, **kw):
    p = abi.default_physics(*dims)
    p.mode = 1
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_default_physics_from_the_library(abi):
    """fireCudaDefaultPhysicsParams is host-only: mode 0, the reference's buoyancy constants."""
    p = abi.default_physics(64, 48, 80)
    assert p.mode == 0 and p.emitterCount == 0
    assert p.buoyancyHeat == pytest.approx(1.62) and p.buoyancySoot == pytest.approx(0.095)
    assert p.dt == pytest.approx(1 / 60)
    assert (p.targetX, p.targetY, p.targetZ) == (32.0, 24.0, 40.0)
    assert p.eyeZ < 0 and 1 <= p.primarySamples <= 4096 and 1 <= p.lightSamples <= 4096


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_config_workloads_state_their_parameters(abi, name):
    w = abi.config_workload(name)
    p = w["physics"]
    n = w["grid"][0]
    assert p.mode == 1 and p.vorticityEps == pytest.approx(0.3)
    assert p.buoyancySoot == pytest.approx(0.1) and p.buoyancyHeat == pytest.approx(1.0)
    assert p.burnRate == pytest.approx(0.5) and p.sootYield == pytest.approx(0.3)
    if name == "c1":
        assert n == 64 and w["sor"] == (40, 1.7) and p.emitterCount == 1
        e = p.emitters[0]
        assert (e.centerX, e.centerY, e.centerZ, e.radius, e.seed) == (32, 4, 32, 6, 1)
        assert (p.primarySamples, p.lightSamples, p.lightY) == (64, 32, 90)
    elif name == "c2":
        assert n == 128 and w["sor"] == (60, 1.8) and p.windX == pytest.approx(0.5)
        assert (p.noiseSeed, p.noisePeriod) == (7, 16.0) and p.noiseAmplitude == pytest.approx(0.4)
        assert p.emitters[0].radius == 12 and (p.primarySamples, p.lightSamples) == (128, 48)
    else:
        assert n == 256 and w["precision"] == "bf16" and w["tolerance"] == 1e-5 and w["sor"] == (120, 1.85)
        assert p.emitterCount == 2 and [p.emitters[i].radius for i in range(2)] == [16, 10]
        assert all(p.emitters[i].seed == 3 for i in range(2))


def test_emitters_inject_jittered_fuel_on_their_disks(abi, oracle_mod):
    """One ADVECT_REACT from an empty scene: the disk cells of the emitter row hold
    fuel * (1 - jitterScale * U) with U from SplitMix64 of (seed, step, cell)
    (restated here in Python integers); every other cell stays 0."""
    dims = (20, 12, 18)
    p = _physics(abi, dims, ignitionHeat=10.0, cooling=0.0)
    p.emitterCount = 2
    p.emitters[0] = abi.FireEmitterDisk(centerX=6.0, centerY=2.0, centerZ=7.5, radius=3.2, fuel=1.0, heat=0.9,
                                        upVelocity=2.0, jitterScale=0.2, seed=1)
    p.emitters[1] = abi.FireEmitterDisk(centerX=15.0, centerY=5.7, centerZ=12.0, radius=2.0, fuel=0.5, heat=0.7,
                                        upVelocity=1.0, jitterScale=0.5, seed=99)
    o = _oracle(abi, oracle_mod, dims, p)
    for step in range(3):
        o.stages("advect_react", "advect_react")
        fuel, heat = o.get("fuel"), o.get("heat")
        want_f = np.zeros_like(fuel)
        want_h = np.zeros_like(heat)
        for e in (p.emitters[0], p.emitters[1]):
            row, inside = disk_cells(*dims, e)
            for z, x in zip(*np.nonzero(inside)):
                cell = (z * dims[1] + row) * dims[0] + x
                j = np.float32(1) - np.float32(e.jitterScale) * jitter(e.seed, step, int(cell))
                want_f[z, row, x] = max(want_f[z, row, x], np.float32(e.fuel) * j)
                want_h[z, row, x] = max(want_h[z, row, x], np.float32(e.heat) * j)
        # Without velocity the backtrace returns each cell to itself: the fields only grow to the new maximum.
        if step == 0:
            np.testing.assert_array_equal(fuel, want_f)
            np.testing.assert_array_equal(heat, want_h)
        else:
            np.testing.assert_array_equal(fuel, np.maximum(prev_f, want_f))
        prev_f = fuel
    assert o.step_count() == 3


def test_burn_decay_and_soot_yield(abi, oracle_mod):
    """One reaction step in a still scene: burn = F * min(1, rate * dt) where
    T > ignition; T and S decay by their rates."""
    dims = (8, 6, 5)
    p = _physics(abi, dims, burnRate=0.5, ignitionHeat=0.5, heatRelease=2.0, sootYield=0.3, cooling=0.6, sootDecay=0.1)
    o = _oracle(abi, oracle_mod, dims, p)
    rng = np.random.default_rng(1)
    heat = rng.uniform(0, 1, (5, 6, 8)).astype(np.float32)
    fuel = rng.uniform(0, 1, (5, 6, 8)).astype(np.float32)
    soot = rng.uniform(0, 0.2, (5, 6, 8)).astype(np.float32)
    for n, a in (("heat", heat), ("fuel", fuel), ("soot", soot)):
        o.set(n, a)
    o.stages("advect_react", "advect_react")
    f = np.float32
    dt = f(p.dt)
    burn = np.where(heat > f(0.5), fuel * min(f(1), f(0.5) * dt), f(0))
    h = np.where(heat > f(0.5), heat + f(2.0) * burn, heat)
    s = np.where(heat > f(0.5), soot + f(0.3) * burn, soot)
    np.testing.assert_array_equal(o.get("fuel"), np.where(heat > f(0.5), fuel - burn, fuel))
    np.testing.assert_array_equal(o.get("heat"), h - h * min(f(1), f(0.6) * dt))
    np.testing.assert_array_equal(o.get("soot"), s - s * min(f(1), f(0.1) * dt))


def _divergence(u, v, w):
    return (u[:, :, 1:] - u[:, :, :-1]) + (v[:, 1:, :] - v[:, :-1, :]) + (w[1:] - w[:-1])


def test_projection_removes_most_divergence(abi, oracle_mod):
    """A step of the C1 physics at 32^3: the projected velocity's divergence is
    far below the forced velocity's, and the walls hold."""
    dims = (32, 32, 32)
    w = abi.config_workload("c1")
    p = w["physics"]
    p.emitters[0].centerX, p.emitters[0].centerZ, p.emitters[0].radius = 16, 16, 4
    o = _oracle(abi, oracle_mod, dims, p)
    o.set_pressure_solver(200, 1.8)
    for _ in range(6):
        o.step()
    o.stages("advect_velocity", "force")
    before = np.abs(_divergence(o.get("u"), o.get("v"), o.get("w"))[:-1]).max()
    o.stages("divergence", "wall_boundary")
    u, v, ww = o.get("u"), o.get("v"), o.get("w")
    after = np.abs(_divergence(u, v, ww)[:-1]).max()  # below the open top row
    assert before > 0.1 and after < 0.05 * before, (before, after)
    assert not u[:, :, 0].any() and not u[:, :, -1].any() and not v[:, 0, :].any()
    assert not ww[0].any() and not ww[-1].any()


def test_float_oracle_tracks_the_double_oracle(abi, oracle_mod):
    """20 steps of a C2-like scene at 32^3 with noise, wind and confinement: the
    float restatement stays within 1e-4 relative L2 of the double one."""
    dims = (32, 32, 32)
    w = abi.config_workload("c2")
    p = w["physics"]
    p.emitters[0].centerX, p.emitters[0].centerY, p.emitters[0].centerZ, p.emitters[0].radius = 16, 3, 16, 5
    p.noisePeriod = 8.0
    outs = []
    for prec in ("f32", "f64"):
        o = _oracle(abi, oracle_mod, dims, p, precision=prec)
        o.set_pressure_solver(40, 1.8)
        for _ in range(20):
            o.step()
        outs.append({n: o.get64(n) for n in ("heat", "fuel", "soot", "u", "v", "w")})
    for n in outs[0]:
        a, b = outs[0][n], outs[1][n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 1e-4, (n, rel)
    assert outs[1]["heat"].sum() > 10.0


def _mg_oracle(abi, oracle_mod, dims, cycles, tol, seed=2):
    o = oracle_mod.ConfigOracle(abi, 16, 16, *dims)
    p = abi.default_physics(*dims)
    p.mode, p.pressureTop = 1, 1
    o.set_physics(p)
    d = (0.3 * np.random.default_rng(seed).standard_normal(dims[::-1])).astype(np.float32)
    o.set("divergence", d)
    o.set("pressure", np.zeros(dims[::-1], np.float32))
    o.set_multigrid(cycles, 2, 2, tol)
    return o, d


def _residual_dirichlet_top(p, d):
    """d + (neighbours: the cell itself at walls and floor, -p above the top row) - 6p, in float64."""
    p = p.astype(np.float64)
    pad = np.pad(p, 1, mode="edge")
    pad[1:-1, -1, 1:-1] = -p[:, -1, :]
    nb = (pad[1:-1, 1:-1, :-2] + pad[1:-1, 1:-1, 2:] + pad[1:-1, :-2, 1:-1] + pad[1:-1, 2:, 1:-1] + pad[:-2, 1:-1, 1:-1] +
          pad[2:, 1:-1, 1:-1])
    return d + nb - 6.0 * p


@pytest.mark.parametrize("dims,max_cycles", [((32, 32, 32), 8), ((64, 48, 40), 8), ((48, 24, 40), 8)])
def test_multigrid_converges(abi, oracle_mod, dims, max_cycles):
    """Semi-coarsening V-cycles with the Dirichlet top reach max |r| <= 1e-5 in a
    few cycles (about a factor 6 per cycle), and the reported residual is the
    residual of the returned pressure."""
    o, d = _mg_oracle(abi, oracle_mod, dims, 40, 1e-5)
    o.stages("pressure_sor", "pressure_sor")
    cycles, max_r = o.multigrid_stats()
    assert cycles <= max_cycles and max_r <= 1e-5, (cycles, max_r)
    # The float residual near 1e-5 carries the rounding of its O(|p|) terms (a few 1e-7 each).
    r = _residual_dirichlet_top(o.get("pressure"), d)
    assert np.abs(r).max() == pytest.approx(max_r, abs=2e-6)


def test_multigrid_odd_extents_stay_stable(abi, oracle_mod):
    """Odd extents are not coarsened: the solve degrades to the smoother but
    still decreases the residual monotonically over cycles."""
    prev = None
    for cycles in (2, 6, 12):
        o, d = _mg_oracle(abi, oracle_mod, (33, 17, 21), cycles, 0.0)
        o.stages("pressure_sor", "pressure_sor")
        m = float(np.abs(_residual_dirichlet_top(o.get("pressure"), d)).max())
        assert prev is None or m < prev
        prev = m


def test_config_projection_meets_the_divergence_bound(abi, oracle_mod):
    """Config physics with the Dirichlet top and the multigrid solve at max |r|
    <= 1e-5: after every projection of 6 steps the velocity's divergence
    (every cell, top faces included) is below 1e-4."""
    dims = (32, 32, 32)
    w = abi.config_workload("c1")
    p = w["physics"]
    p.emitters[0].centerX, p.emitters[0].centerZ, p.emitters[0].radius = 16, 16, 4
    p.pressureTop = 1
    o = oracle_mod.ConfigOracle(abi, 16, 16, *dims)
    o.set_physics(p)
    o.set_multigrid(30, 2, 2, 1e-5)
    for _ in range(6):
        o.step()
        div = _divergence(o.get("u"), o.get("v"), o.get("w"))
        assert np.abs(div).max() <= 1e-4, np.abs(div).max()
    assert o.get("heat").sum() > 1.0
