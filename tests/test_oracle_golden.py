"""Pins the CPU oracle against the reference itself.

The fixtures in tests/golden/ were recorded from native-firesim's own CUDA code
(src/fire_cuda.cu compiled unmodified for sm_100a, run on a B200 by
tests/golden/make_golden.py).  Each test feeds the oracle exactly the inputs
the reference saw and compares outputs under the tolerance classes of
tests/tolerances.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import RENDER_STAGES, STAGE_OUTPUTS, STATE_FIELDS
import tolerances as T

STAGES = list(STAGE_OUTPUTS)


def _oracle(oracle_mod, abi, meta):
    nx, ny, nz = meta["grid"]
    fw, fh = meta["frame"]
    o = oracle_mod.OracleFire(abi, fw, fh, nx, ny, nz)
    assert list(o.light_dims) == meta["light"]
    return o


@pytest.mark.parametrize("stage", STAGES)
def test_validation_chain_stage(stage, oracle_mod, abi, golden):
    """Frame 11 of the validation harness, stage by stage (input = the reference's previous stage)."""
    data, meta = golden("validation_s0")
    o = _oracle(oracle_mod, abi, meta)
    settings = abi.FireSettings(**meta["chain"]["settings"])
    state = {n: data[f"pre/{n}"] for n in STATE_FIELDS}
    for prior in STAGES[: STAGES.index(stage)]:
        for n in STAGE_OUTPUTS[prior]:
            state[n] = data[f"chain/{prior}/{n}"]
    for n, a in state.items():
        if n in ("hdr", "bgra") or n in STATE_FIELDS:
            o.set(n, a)
    time = meta["chain"]["render_time"] if stage in RENDER_STAGES else meta["chain"]["sim_time"]
    o.stages(stage, stage, settings, time)
    for n in STAGE_OUTPUTS[stage]:
        ref = data[f"chain/{stage}/{n}"]
        if n == "bgra":
            T.check_bgra(f"{stage}/{n}", o.get(n), ref, max_lsb=1, max_frac=0.01)
        else:
            T.check_field(f"{stage}/{n}", o.get(n), ref, T.stage_tol(stage, n))
    if stage == "metrics":
        sums, words = o.last_metrics()
        rs, rw = data["chain/metrics/sums"], data["chain/metrics/bits"]
        np.testing.assert_allclose(sums, rs, rtol=1e-6, atol=1e-9)
        np.testing.assert_array_equal(words, rw)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("stage", STAGES)
def test_random_state_stage(stage, variant, oracle_mod, abi, golden):
    """Every stage from one seeded random state on an odd 17x21x11 grid, three settings variants."""
    data, meta = golden("random")
    o = _oracle(oracle_mod, abi, meta)
    settings = abi.FireSettings(**meta["variants"][variant])
    inputs = {k[3:]: data[k] for k in data.files if k.startswith("in/")}
    for n, a in inputs.items():
        o.set(n, a)
    o.stages(stage, stage, settings, meta["time"])
    for n in STAGE_OUTPUTS[stage]:
        ref = data[f"v{variant}/{stage}/{n}"]
        if n == "bgra":
            T.check_bgra(f"{stage}/{n}", o.get(n), ref, max_lsb=1, max_frac=0.01)
        else:
            T.check_field(f"v{variant}/{stage}/{n}", o.get(n), ref, T.stage_tol(stage, n))
    if stage == "metrics":
        sums, words = o.last_metrics()
        np.testing.assert_allclose(sums, data[f"v{variant}/metrics/sums"], rtol=1e-6, atol=1e-9)
        np.testing.assert_array_equal(words, data[f"v{variant}/metrics/bits"])


@pytest.mark.parametrize("mode", range(1, 7))
def test_render_debug_modes(mode, oracle_mod, abi, golden):
    data, meta = golden("random")
    o = _oracle(oracle_mod, abi, meta)
    settings = abi.FireSettings(**meta["variants"][0])
    settings.renderDebugMode = mode
    for k in data.files:
        if k.startswith("in/"):
            o.set(k[3:], data[k])
    o.stages("render", "render", settings, meta["time"])
    T.check_field(f"render_debug{mode}", o.get("hdr"), data[f"v0/render_debug{mode}/hdr"], T.SATURATED)


@pytest.mark.parametrize("scene", [1, 2])
def test_scene_reset(scene, oracle_mod, abi, golden):
    """Procedural fuel beds of the campfire and burner scenes (src/fire_cuda.cu:746-848)."""
    data, meta = golden(f"scene{scene}")
    o = _oracle(oracle_mod, abi, meta)
    o.stages("reset", "reset", abi.FireSettings(**meta["reset"]["settings"]), meta["reset"]["time"])
    for n in STATE_FIELDS[:10]:
        T.check_field(f"scene{scene}/reset/{n}", o.get(n), data[f"reset/{n}"], T.NOISE)
    for n in ("u", "v", "w", "pressure"):
        assert np.all(o.get(n) == data[f"reset/{n}"])


def _check_state(tag, o, data, prefix):
    for n in STATE_FIELDS:
        tol = T.TRAJECTORY_LIGHT if n == "scene_light" else T.TRAJECTORY
        T.check_field(f"{tag}/{n}", o.get(n), data[f"{prefix}/{n}"], tol)
    T.check_field(f"{tag}/hdr", o.get("hdr"), data[f"{prefix}/hdr"], T.TRAJECTORY)


@pytest.mark.parametrize("scene", [1, 2])
def test_scene_trajectory(scene, oracle_mod, abi, golden):
    """Three whole frames (reset on frame 0) through oracle_step vs stepAndRenderInternal."""
    data, meta = golden(f"scene{scene}")
    o = _oracle(oracle_mod, abi, meta)
    for f in range(3):
        bgra, metrics = o.step(abi.FireSettings(**meta["frames"][str(f)]["settings"]), mode=1)
        assert list(o.times()) == pytest.approx(meta["frames"][str(f)]["times"], abs=0)
    _check_state(f"scene{scene}", o, data, "f2")
    T.check_bgra(f"scene{scene}/bgra", bgra, data["f2/bgra"], max_lsb=3, max_frac=0.2)


def _check_metrics(tag, metrics, data, prefix):
    keys = [str(k) for k in data[f"{prefix}metrics_keys"]]
    ref = dict(zip(keys, data[f"{prefix}metrics"]))
    got = metrics.as_dict()
    for k in ("frameIndex", "gridX", "gridY", "gridZ", "pressureIterations", "invalidCells"):
        assert got[k] == ref[k], (tag, k)
    assert got["timeSeconds"] == pytest.approx(ref["timeSeconds"], abs=0)
    for k, v in ref.items():
        if k in ("meanSceneLight", "meanRoomIrradiance", "meanVolumetricShadow"):
            assert got[k] == pytest.approx(v, rel=0.05, abs=1e-7), (tag, k)
        else:
            assert got[k] == pytest.approx(v, rel=0.02, abs=1e-5), (tag, k)


def test_validation_trajectory(oracle_mod, abi, golden):
    """Frames 0..10 of the validation harness (reset on frame 0), compared at frames 0 and 5."""
    data, meta = golden("validation_s0")
    o = _oracle(oracle_mod, abi, meta)
    for f in range(11):
        bgra, metrics = o.step(abi.FireSettings(**meta["frames"][str(f)]["settings"]), mode=1)
        assert list(o.times()) == pytest.approx(meta["frames"][str(f)]["times"], abs=0)
        if f in (0, 5):
            _check_state(f"f{f}", o, data, f"f{f}")
            T.check_bgra(f"f{f}/bgra", bgra, data[f"f{f}/bgra"], max_lsb=3, max_frac=0.2)
            _check_metrics(f"f{f}", metrics, data, f"f{f}/")


def test_whole_step_from_state(oracle_mod, abi, golden):
    """One whole frame (oracle_step) from the reference's state after frame 10."""
    data, meta = golden("validation_s0")
    o = _oracle(oracle_mod, abi, meta)
    for n in STATE_FIELDS:
        o.set(n, data[f"pre/{n}"])
    t = meta["frames"]["10"]["times"]
    o.set_times(t[0], t[1], t[2])
    bgra, metrics = o.step(abi.FireSettings(**meta["chain"]["settings"]), mode=1)
    for n in STATE_FIELDS:
        tol = {"scene_light": T.SATURATED}.get(n, T.NOISE if n not in ("pressure", "divergence", "u", "v", "w")
                                               else T.Tol(5e-3, 2e-3, 0.9))
        T.check_field(f"step11/{n}", o.get(n), data[f"step11/{n}"], tol)
    T.check_field("step11/hdr", o.get("hdr"), data["step11/hdr"], T.NOISE)
    T.check_bgra("step11/bgra", bgra, data["step11/bgra"], max_lsb=1, max_frac=0.03)
    _check_metrics("step11", metrics, data, "step11/")


def test_double_oracle_tracks_float(oracle_mod, abi, golden):
    """The FP64 instantiation stays close to the FP32 one over the validation frames."""
    data, meta = golden("validation_s0")
    nx, ny, nz = meta["grid"]
    fw, fh = meta["frame"]
    of = oracle_mod.OracleFire(abi, fw, fh, nx, ny, nz, "f32")
    od = oracle_mod.OracleFire(abi, fw, fh, nx, ny, nz, "f64")
    for f in range(6):
        s = abi.FireSettings(**meta["frames"][str(f)]["settings"])
        of.step(s, mode=2)
        od.step(s, mode=2)
    for n in ("heat", "fuel", "soot", "u", "v", "w", "pressure"):
        st = T.field_stats(of.get(n), od.get64(n))
        assert st["rel_l2"] < 5e-2, (n, st)
