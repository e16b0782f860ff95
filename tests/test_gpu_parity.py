"""Parity of the sm_100a product against the reference and the oracle (needs a B200).

Three comparisons:
  * product vs the reference's own CUDA outputs recorded in tests/golden/
    (GPU against GPU: same device sinf, so classes GPU_EXACT / GPU_NOISE);
  * product vs the CPU oracle on identical inputs (statistical classes, as the
    oracle-pin tests);
  * product vs the live reference kernels (oracle/_ref) on fresh random states
    at other grid shapes.
Every product call goes through the C ABI of libfiresim_b200.so.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import RENDER_STAGES, STAGE_OUTPUTS, STATE_FIELDS
import tolerances as T

pytestmark = pytest.mark.gpu

STAGES = list(STAGE_OUTPUTS)

# GPU-vs-GPU classes.  Most stages are bit-identical to the reference's own
# kernels (the tolerance only has to absorb nothing).  force carries the
# reference's atomic-add order.  render matches the reference's renderKernel
# to float rounding (GPU_EXACT): its fbm3 calls are compiled out of line there,
# with the sin hash evaluated in plain (uncontracted) form, and the product's
# raymarch evaluates them the same way (renderFbm3); the CPU oracle follows
# the source definition.
# The stages whose arithmetic is all correctly rounded (no sin hash, no atomic
# order) are the reference's bits; the others keep a statistical class.
GPU_CLASS = {
    "advect_velocity": T.BITS, "advect_react": T.GPU_NOISE, "force": T.GPU_NOISE,
    "velocity_boundary": T.BITS, "divergence": T.BITS, "pressure_sor": T.BITS,
    "subtract": T.BITS, "wall_boundary": T.BITS, "light_build": T.GPU_NOISE,
    "light_propagate": T.BITS, "render": T.GPU_EXACT, "embers": T.GPU_NOISE, "metrics": T.GPU_EXACT,
}


@pytest.fixture(scope="module")
def product(pkg):
    return pkg


def _sim(pkg, meta):
    nx, ny, nz = meta["grid"]
    fw, fh = meta["frame"]
    sim = pkg.FireSim(fw, fh, nx, ny, nz)
    assert list(sim.light_dims) == meta["light"]
    return sim


def _compare(tag, got, ref, tol):
    if got.dtype == np.uint32:
        T.check_bgra(tag, got, ref, max_lsb=1, max_frac=0.01)
    else:
        T.check_field(tag, got, ref, tol)


@pytest.mark.parametrize("stage", STAGES)
def test_stage_vs_reference_chain(stage, product, abi, golden):
    """Validation frame 11, one stage at a time, from the reference's own previous-stage output."""
    data, meta = golden("validation_s0")
    sim = _sim(product, meta)
    settings = abi.FireSettings(**meta["chain"]["settings"])
    state = {n: data[f"pre/{n}"] for n in STATE_FIELDS}
    for prior in STAGES[: STAGES.index(stage)]:
        for n in STAGE_OUTPUTS[prior]:
            state[n] = data[f"chain/{prior}/{n}"]
    for n, a in state.items():
        sim.set(n, a)
    time = meta["chain"]["render_time"] if stage in RENDER_STAGES else meta["chain"]["sim_time"]
    sim.stages(stage, stage, settings, time)
    for n in STAGE_OUTPUTS[stage]:
        _compare(f"{stage}/{n}", sim.get(n), data[f"chain/{stage}/{n}"], GPU_CLASS.get(stage, T.GPU_EXACT))


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("stage", STAGES)
def test_stage_vs_reference_random(stage, variant, product, abi, golden):
    """Every stage from the seeded random state (odd 17x21x11 grid), three settings variants."""
    data, meta = golden("random")
    sim = _sim(product, meta)
    settings = abi.FireSettings(**meta["variants"][variant])
    inputs = {k[3:]: data[k] for k in data.files if k.startswith("in/")}
    for n, a in inputs.items():
        sim.set(n, a)
    sim.stages(stage, stage, settings, meta["time"])
    for n in STAGE_OUTPUTS[stage]:
        tol = GPU_CLASS.get(stage, T.GPU_EXACT)
        _compare(f"v{variant}/{stage}/{n}", sim.get(n), data[f"v{variant}/{stage}/{n}"], tol)


@pytest.mark.parametrize("stage", STAGES)
def test_stage_vs_oracle(stage, product, abi, golden, oracle_mod):
    """Product and CPU oracle from the same random state."""
    data, meta = golden("random")
    sim = _sim(product, meta)
    nx, ny, nz = meta["grid"]
    fw, fh = meta["frame"]
    o = oracle_mod.OracleFire(abi, fw, fh, nx, ny, nz)
    settings = abi.FireSettings(**meta["variants"][1])
    for k in data.files:
        if k.startswith("in/"):
            sim.set(k[3:], data[k])
            o.set(k[3:], data[k])
    sim.stages(stage, stage, settings, meta["time"])
    o.stages(stage, stage, settings, meta["time"])
    for n in STAGE_OUTPUTS[stage]:
        if n == "bgra":
            T.check_bgra(f"{stage}/{n}", sim.get(n), o.get(n), max_lsb=1, max_frac=0.01)
        else:
            T.check_field(f"{stage}/{n}", sim.get(n), o.get(n), T.stage_tol(stage, n))


@pytest.mark.parametrize("mode", range(1, 7))
def test_render_debug_modes(mode, product, abi, golden):
    data, meta = golden("random")
    sim = _sim(product, meta)
    settings = abi.FireSettings(**meta["variants"][0])
    settings.renderDebugMode = mode
    for k in data.files:
        if k.startswith("in/"):
            sim.set(k[3:], data[k])
    sim.stages("render", "render", settings, meta["time"])
    T.check_field(f"debug{mode}", sim.get("hdr"), data[f"v0/render_debug{mode}/hdr"], T.GPU_EXACT)


def test_fused_ranges_match_single_stages(product, abi, golden):
    """The fused kernels (force+boundary+divergence, subtract+walls, tonemap+overlay)
    equal the stage-by-stage path exactly."""
    data, meta = golden("random")
    settings = abi.FireSettings(**meta["variants"][1])
    inputs = {k[3:]: data[k] for k in data.files if k.startswith("in/")}
    sim = _sim(product, meta)
    out = {}
    for ranges in ([("force", "divergence"), ("subtract", "wall_boundary"), ("tonemap", "overlay")],
                   [(s, s) for s in ("force", "velocity_boundary", "divergence")] + [("subtract", "subtract"),
                    ("wall_boundary", "wall_boundary"), ("tonemap", "tonemap"), ("overlay", "overlay")]):
        for n, a in inputs.items():
            sim.set(n, a)
        for first, last in ranges:
            sim.stages(first, last, settings, meta["time"])
        out[len(ranges)] = {n: sim.get(n) for n in ("u", "v", "w", "divergence", "pressure", "bgra")}
    a, b = out.values()
    for n in a:
        np.testing.assert_array_equal(a[n], b[n], err_msg=n)


def test_frames_vs_reference_trajectory(product, abi, golden):
    """Frames 0..10 of the validation harness through fireCudaStepAndRenderMeasured."""
    data, meta = golden("validation_s0")
    sim = _sim(product, meta)
    for f in range(11):
        bgra, metrics = sim.step_and_render(abi.FireSettings(**meta["frames"][str(f)]["settings"]), metrics=True)
        assert list(sim.times()) == pytest.approx(meta["frames"][str(f)]["times"], abs=0)
        if f in (0, 5):
            for n in STATE_FIELDS:
                tol = T.TRAJECTORY_LIGHT if n == "scene_light" else T.TRAJECTORY
                T.check_field(f"f{f}/{n}", sim.get(n), data[f"f{f}/{n}"], tol)
            T.check_bgra(f"f{f}/bgra", bgra, data[f"f{f}/bgra"], max_lsb=3, max_frac=0.2)
            keys = [str(k) for k in data[f"f{f}/metrics_keys"]]
            ref = dict(zip(keys, data[f"f{f}/metrics"]))
            got = metrics.as_dict()
            for k in ("frameIndex", "gridX", "gridY", "gridZ", "pressureIterations", "invalidCells"):
                assert got[k] == ref[k], k
            for k in ("heatSum", "fuelSum", "sootSum", "charSum", "divergenceBeforeL2", "divergenceAfterL2", "maxHeat"):
                assert got[k] == pytest.approx(ref[k], rel=0.02, abs=1e-5), k


def test_whole_step_vs_reference(product, abi, golden):
    """One whole frame from the reference's state after frame 10."""
    data, meta = golden("validation_s0")
    sim = _sim(product, meta)
    for n in STATE_FIELDS:
        sim.set(n, data[f"pre/{n}"])
    t = meta["frames"]["10"]["times"]
    sim.set_times(t[0], t[1], t[2])
    bgra, metrics = sim.step_and_render(abi.FireSettings(**meta["chain"]["settings"]), metrics=True)
    for n in STATE_FIELDS:
        tol = {"scene_light": T.SATURATED}.get(n, T.GPU_NOISE)
        T.check_field(f"step11/{n}", sim.get(n), data[f"step11/{n}"], tol)
    T.check_field("step11/hdr", sim.get("hdr"), data["step11/hdr"], T.NOISE)
    T.check_bgra("step11/bgra", bgra, data["step11/bgra"], max_lsb=1, max_frac=0.03)


@pytest.mark.parametrize("scene", [1, 2])
def test_scene_reset_and_frames(scene, product, abi, golden):
    data, meta = golden(f"scene{scene}")
    sim = _sim(product, meta)
    sim.stages("reset", "reset", abi.FireSettings(**meta["reset"]["settings"]), meta["reset"]["time"])
    for n in STATE_FIELDS[:10]:
        T.check_field(f"scene{scene}/reset/{n}", sim.get(n), data[f"reset/{n}"], T.GPU_EXACT)
    sim2 = _sim(product, meta)
    for f in range(3):
        bgra, _ = sim2.step_and_render(abi.FireSettings(**meta["frames"][str(f)]["settings"]), metrics=True)
    for n in STATE_FIELDS:
        tol = T.TRAJECTORY_LIGHT if n == "scene_light" else T.TRAJECTORY
        T.check_field(f"scene{scene}/f2/{n}", sim2.get(n), data[f"f2/{n}"], tol)


def test_deterministic(product, abi):
    """Two runs of the same frames are bit-identical (no atomics in the step)."""
    outs = []
    for _ in range(2):
        sim = product.FireSim(64, 40, 24, 28, 20)
        for f in range(6):
            s = abi.validation_settings(f, width=64, height=40)
            bgra, _ = sim.step_and_render(s)
        outs.append({n: sim.get(n) for n in STATE_FIELDS + ["hdr"]} | {"bgra": bgra})
    for n in outs[0]:
        np.testing.assert_array_equal(outs[0][n], outs[1][n], err_msg=n)


@pytest.mark.parametrize("dims", [(17, 21, 11), (64, 64, 64), (128, 128, 128), (40, 34, 70)])
def test_sor_resident_equals_per_launch(dims, product, abi):
    """The shared-memory-resident SOR (one cooperative launch) equals the
    colour-split path (one graph of per-half-sweep launches) bit for bit."""
    nx, ny, nz = dims
    rng = np.random.default_rng(nx * 7 + ny)
    p0 = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    d0 = (0.3 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    s = abi.FireSettings()
    out = []
    for path in (1, 2):
        sim = product.FireSim(32, 16, nx, ny, nz)
        sim.set_pressure_solver(60, 1.8)
        sim.set_pressure_path(path)
        sim.set("pressure", p0)
        sim.set("divergence", d0)
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
        first = sim.get("pressure")
        assert sim.pressure_path_used() == path
        # A second solve in the same scene: the neighbour flags' epochs advance.
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
        out.append((first, sim.get("pressure")))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_resident_sor_wait_runs_out_and_reports(product, abi):
    """Failure detection of the resident SOR without a GPU fault: brick 5 is told
    (from the host) never to announce its half sweeps, so its neighbours' waits
    run out after 2 ms; the solve returns, the stage call reports the timed-out
    brick, and the next solve on the same scene is correct again."""
    nx, ny, nz = 64, 64, 64
    rng = np.random.default_rng(11)
    p0 = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    d0 = (0.3 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    s = abi.FireSettings()
    ref = product.FireSim(32, 16, nx, ny, nz)
    ref.set_pressure_solver(20, 1.8)
    ref.set_pressure_path(1)
    ref.set("pressure", p0)
    ref.set("divergence", d0)
    ref.stages("pressure_sor", "pressure_sor", s, 0.0)
    expect = ref.get("pressure")
    ref.close()

    sim = product.FireSim(32, 16, nx, ny, nz)
    sim.set_pressure_solver(20, 1.8)
    sim.set_pressure_path(2)
    sim.set_resident_sor_fault(5, 2000)
    sim.set("pressure", p0)
    sim.set("divergence", d0)
    with pytest.raises(product.firesim.FireSimError, match="timed out waiting for a neighbour"):
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
    sim.synchronize()  # the failure is reported once
    sim.set_resident_sor_fault(-1, 1_000_000)
    sim.set("pressure", p0)
    sim.set("divergence", d0)
    sim.stages("pressure_sor", "pressure_sor", s, 0.0)
    assert sim.pressure_path_used() == 2
    np.testing.assert_array_equal(sim.get("pressure"), expect)


@pytest.mark.parametrize("scene", [0, 1, 2])
def test_hash_lattices_equal_in_place_hashing(scene, product, abi):
    """The per-step and per-frame hash tables (curl noise, fuel-bed source noise,
    the raymarch's four fbm3 fields) give the same bits as hashing every corner
    in place: 8 frames with a render each, full state and HDR compared."""
    out = []
    for lattices in (True, False):
        sim = product.FireSim(96, 64, 64, 64, 64)
        sim.set_hash_lattices(lattices)
        frames = []
        for f in range(8):
            s = abi.validation_settings(f, scene=scene, width=96, height=64)
            s.reset = 1 if f == 0 else 0
            bgra, _ = sim.step_and_render(s)
            frames.append((bgra, sim.get("hdr")))
        state = {n: sim.get(n) for n in abi.SCALAR_FIELDS + ["u", "v", "w", "pressure"]}
        out.append((frames, state))
        sim.close()
    for f, (a, b) in enumerate(zip(out[0][0], out[1][0])):
        np.testing.assert_array_equal(a[0], b[0], err_msg=f"bgra frame {f}")
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32), err_msg=f"hdr frame {f}")
    for n in out[0][1]:
        np.testing.assert_array_equal(out[0][1][n].view(np.uint32), out[1][1][n].view(np.uint32), err_msg=n)


@pytest.mark.parametrize("scene", [1, 2])
def test_scene_contract_frames_vs_oracle(scene, product, abi, oracle_mod):
    """The validation harness with the scene's contract applied (the emitter of
    the campfire bed, the selected gas burner): 4 steps on the product and on
    the CPU oracle from the same settings, compared per field in the
    trajectory class."""
    from pathlib import Path
    contracts = Path(__file__).resolve().parent / "golden" / "scene_contracts"
    nx, ny, nz = 32, 36, 24
    sim = product.FireSim(48, 32, nx, ny, nz)
    o = oracle_mod.OracleFire(abi, 48, 32, nx, ny, nz)
    for f in range(4):
        s = abi.validation_settings(f, scene=scene, width=48, height=32, fire_scenes_dir=contracts)
        assert s.burnerCenterCount == (1 if scene == 2 else 0)
        sim.step(s)
        o.step(s, mode=2)  # advance without rendering, as fireCudaStepD3D11
    sim.synchronize()
    for n in STATE_FIELDS[:10] + ["u", "v", "w"]:
        T.check_field(f"contract{scene}/{n}", sim.get(n), o.get(n), T.TRAJECTORY)
    assert sim.get("heat").sum() > 0.0



def _residual(p, d):
    """r = d + (six neighbours, clamped) - 6p in float32, summed in the kernel's order; max |r| and FP64 L2."""
    f = np.float32
    pad = np.pad(p, 1, mode="edge")
    nb = [pad[1:-1, 1:-1, :-2], pad[1:-1, 1:-1, 2:], pad[1:-1, :-2, 1:-1], pad[1:-1, 2:, 1:-1], pad[:-2, 1:-1, 1:-1], pad[2:, 1:-1, 1:-1]]
    acc = d.astype(f)
    for n in nb:
        acc = (acc + n).astype(f)
    r = (acc - f(6.0) * p).astype(f)
    return float(np.abs(r).max()), float(np.sqrt(np.sum(r.astype(np.float64) ** 2)))


@pytest.mark.parametrize("pressure_path", [1, 2])
def test_pressure_tolerance_gates_the_solve(pressure_path, product, abi):
    """The residual-gated solve stops at the first check with max |r| <= tolerance,
    and its result equals a fixed solve of the same iteration count; a tolerance
    never reached runs every iteration and equals the fixed solve.  Both solve
    paths: resident (2) and colour-split (1)."""
    nx, ny, nz = 64, 48, 40
    rng = np.random.default_rng(5)
    p0 = np.zeros((nz, ny, nx), np.float32)
    d0 = (0.2 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    d0 -= d0.mean()
    s = abi.FireSettings()

    def solve(iters, tol, every=10):
        sim = product.FireSim(32, 16, nx, ny, nz)
        sim.set_pressure_solver(iters, 1.8)
        sim.set_pressure_path(pressure_path)
        sim.set_pressure_tolerance(tol, every)
        sim.set("pressure", p0)
        sim.set("divergence", d0)
        sim.stages("pressure_sor", "pressure_sor", s, 0.0)
        out = sim.get("pressure"), sim.pressure_stats(), sim.pressure_path_used()
        sim.close()
        return out

    fixed, stats, path = solve(120, 0.0)
    assert path == pressure_path and stats[0] == 120 and stats[1] == -1.0
    never, stats_never, _ = solve(120, 1e-30)
    assert stats_never[0] == 120
    np.testing.assert_array_equal(never.view(np.uint32), fixed.view(np.uint32))
    mx_ref, l2_ref = _residual(never, d0)
    assert stats_never[1] == mx_ref
    assert stats_never[2] == pytest.approx(l2_ref, rel=1e-6)
    # A reachable tolerance: the residual after 40 iterations.
    at40, _, _ = solve(40, 0.0)
    tol = _residual(at40, d0)[0] * 1.01
    gated, stats_gated, _ = solve(120, tol)
    m = stats_gated[0]
    assert m % 10 == 0 and m <= 40 and stats_gated[1] <= tol
    fixed_m, _, _ = solve(m, 0.0)
    np.testing.assert_array_equal(gated.view(np.uint32), fixed_m.view(np.uint32))
