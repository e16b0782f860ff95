"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs native-firesim's own CUDA code (oracle/_ref/libfire_ref.so, built by
oracle/build_ref.py from src/fire_cuda.cu) on a GPU and records its inputs and
outputs as compressed .npz files.  The CPU oracle is then pinned against these
files by tests/test_oracle_golden.py, and the product is checked against them
by the GPU tests.

Cases
  validation_s0   scene 0, 20x24x12 grid, 64x40 frame: frames 0..11 of the
                  reference's validation harness (src/main.cpp:4284-4311)
                  through the reference's own stepAndRenderInternal, plus the
                  stage-by-stage chain of frame 11 from the state after frame 10.
  scene1, scene2  reset + 3 validation frames of scenes 1 and 2 (scene 2 with
                  two burner centres), 16x20x12 grid, 48x32 frame.
  random_*        one seeded random state on an odd 17x21x11 grid; every stage
                  is run once from that same state under three settings
                  variants (mouse sources, wind, scenes, render debug modes).

Usage (on a GPU box): python tests/golden/make_golden.py OUTDIR
"""
from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))


def load_abi():
    spec = importlib.util.spec_from_file_location("firesim_abi", ROOT / "native-firesim_b200" / "abi.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


abi = load_abi()
import ref as refmod  # noqa: E402

STATE_FIELDS = abi.SCALAR_FIELDS + ["pressure", "divergence", "u", "v", "w", "scene_light", "scene_shadow"]
STAGE_OUTPUTS = {
    "advect_velocity": ["u", "v", "w"],
    "advect_react": abi.SCALAR_FIELDS,
    "force": ["u", "v", "w"],
    "velocity_boundary": ["u", "v", "w"],
    "divergence": ["divergence", "pressure"],
    "pressure_sor": ["pressure"],
    "subtract": ["u", "v", "w"],
    "wall_boundary": ["u", "v", "w"],
    "light_build": ["scene_light", "scene_shadow"],
    "light_propagate": ["scene_light"],
    "render": ["hdr"],
    "embers": ["hdr"],
    "tonemap": ["bgra"],
    "overlay": ["bgra"],
    "metrics": ["divergence_after"],
}
STAGE_ORDER = list(STAGE_OUTPUTS)


def settings_json(s) -> str:
    return json.dumps(s.as_dict())


def snapshot(ref, names) -> dict:
    return {n: ref.get(n) for n in names}


def save(outdir: Path, name: str, arrays: dict, meta: dict) -> None:
    arrays = dict(arrays)
    arrays["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(outdir / f"{name}.npz", **arrays)
    print(f"wrote {name}.npz ({(outdir / f'{name}.npz').stat().st_size / 1024:.0f} KiB)")


def metrics_arrays(prefix: str, metrics) -> dict:
    d = metrics.as_dict()
    keys = [k for k in d if not k.startswith("gpu")]
    return {f"{prefix}metrics_keys": np.array(keys), f"{prefix}metrics": np.array([d[k] for k in keys], dtype=np.float64)}


def case_validation(outdir: Path) -> None:
    fw, fh, nx, ny, nz = 64, 40, 20, 24, 12
    ref = refmod.RefFire(abi, fw, fh, nx, ny, nz)
    arrays, meta = {}, {"grid": [nx, ny, nz], "frame": [fw, fh], "light": list(ref.light_dims), "frames": {}}
    for frame in range(11):
        s = abi.validation_settings(frame, scene=0, width=fw, height=fh)
        bgra, metrics = ref.step(s, mode=1)
        if frame in (0, 5):
            for n, a in snapshot(ref, STATE_FIELDS + ["hdr"]).items():
                arrays[f"f{frame}/{n}"] = a
            arrays[f"f{frame}/bgra"] = bgra
            arrays.update(metrics_arrays(f"f{frame}/", metrics))
        meta["frames"][str(frame)] = {"settings": s.as_dict(), "times": ref.times()}
    # State after frame 10 = input of the frame-11 chain.
    pre = snapshot(ref, STATE_FIELDS)
    for n, a in pre.items():
        arrays[f"pre/{n}"] = a
    t_sim, t_render, _ = ref.times()
    s11 = abi.validation_settings(11, scene=0, width=fw, height=fh)
    dt = np.float32(s11.dt)
    sim_time = float(np.float32(t_sim) + dt)
    render_time = float(np.float32(t_render) + dt)
    meta["chain"] = {"settings": s11.as_dict(), "sim_time": sim_time, "render_time": render_time}
    for stage in STAGE_ORDER:
        time = render_time if stage in ("render", "embers", "tonemap", "overlay") else sim_time
        ref.stages(stage, stage, s11, time)
        for n in STAGE_OUTPUTS[stage]:
            arrays[f"chain/{stage}/{n}"] = ref.get(n)
        if stage == "metrics":
            sums, bits = ref.last_metrics()
            arrays["chain/metrics/sums"] = sums
            arrays["chain/metrics/bits"] = bits
    # The reference's own full step from the same state, for the harness check
    # and as the whole-step fixture.
    for n, a in pre.items():
        ref.set(n, a)
    bgra, metrics = ref.step(s11, mode=1)
    for n, a in snapshot(ref, STATE_FIELDS + ["hdr"]).items():
        arrays[f"step11/{n}"] = a
    arrays["step11/bgra"] = bgra
    arrays.update(metrics_arrays("step11/", metrics))
    diffs = {}
    for n in STATE_FIELDS:
        chain_last = None
        for stage in reversed(STAGE_ORDER):
            if n in STAGE_OUTPUTS[stage]:
                chain_last = arrays[f"chain/{stage}/{n}"]
                break
        if chain_last is None:
            continue
        diffs[n] = float(np.max(np.abs(chain_last.astype(np.float64) - arrays[f"step11/{n}"])))
    meta["chain_vs_step_maxabs"] = diffs
    print("chain vs step max|diff|:", diffs)
    save(outdir, "validation_s0", arrays, meta)
    ref.close()


def scene_settings(scene: int, frame: int, fw: int, fh: int):
    s = abi.validation_settings(frame, scene=scene, width=fw, height=fh)
    if scene == 1:
        s.emitterRadius = 0.32
        s.emitterHeightNorm = float(np.float32((0.045 - 0.02) / 2.03))
        s.emitterHeightBandNorm = float(np.float32(0.20 / 2.03))
    elif scene == 2:
        s.emitterRadius = 0.24
        s.emitterHeightBandNorm = float(np.float32(0.105 / 2.03))
        s.burnerCenterCount = 2
        for i, (x, y, z) in enumerate([(0.05, 0.138, -0.04), (-0.2, 0.15, 0.1)]):
            s.burnerCenterX[i], s.burnerCenterY[i], s.burnerCenterZ[i] = x, y, z
    return s


def case_scene(outdir: Path, scene: int) -> None:
    fw, fh, nx, ny, nz = 48, 32, 16, 20, 12
    ref = refmod.RefFire(abi, fw, fh, nx, ny, nz)
    arrays, meta = {}, {"grid": [nx, ny, nz], "frame": [fw, fh], "light": list(ref.light_dims), "frames": {}}
    s0 = scene_settings(scene, 0, fw, fh)
    # Reset stage alone, at the time the validation harness's frame 0 uses.
    ref.stages("reset", "reset", s0, float(np.float32(s0.dt)))
    for n, a in snapshot(ref, abi.SCALAR_FIELDS + ["pressure", "divergence", "u", "v", "w"]).items():
        arrays[f"reset/{n}"] = a
    meta["reset"] = {"settings": s0.as_dict(), "time": float(np.float32(s0.dt))}
    for frame in range(3):
        s = scene_settings(scene, frame, fw, fh)
        bgra, metrics = ref.step(s, mode=1)
        meta["frames"][str(frame)] = {"settings": s.as_dict(), "times": ref.times()}
    for n, a in snapshot(ref, STATE_FIELDS + ["hdr"]).items():
        arrays[f"f2/{n}"] = a
    arrays["f2/bgra"] = bgra
    arrays.update(metrics_arrays("f2/", metrics))
    save(outdir, f"scene{scene}", arrays, meta)
    ref.close()


def smooth_field(rng, shape, lo, hi, zero_top=False):
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.linspace(0, 1, nz), np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    f = np.zeros(shape)
    for _ in range(4):
        k = rng.uniform(0.5, 3.0, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        f += rng.uniform(0.2, 1.0) * np.sin(2 * np.pi * k[0] * x + ph[0]) * np.sin(2 * np.pi * k[1] * y + ph[1]) * \
            np.sin(2 * np.pi * k[2] * z + ph[2])
    f = (f - f.min()) / max(1e-9, f.max() - f.min())
    f = lo + (hi - lo) * (0.85 * f + 0.15 * rng.uniform(0, 1, shape))
    if zero_top:
        f = np.where(y > 0.55, 0.0, f)
    return f.astype(np.float32)


def random_state(ref, seed: int) -> dict:
    rng = np.random.default_rng(seed)
    nx, ny, nz = ref.nx, ref.ny, ref.nz
    sh = (nz, ny, nx)
    ranges = {"heat": (0, 3.0), "fuel": (0, 2.0), "oxygen": (0.3, 1.0), "soot": (0, 1.2), "char": (0, 1.5),
              "ash": (0, 0.6), "pyrolysis": (0, 1.0), "progress": (0, 1.5), "turbulence_energy": (0, 1.0),
              "soot_optics": (0, 1.2)}
    st = {}
    for n, (lo, hi) in ranges.items():
        st[n] = smooth_field(rng, sh, lo, hi, zero_top=n not in ("oxygen",))
    st["u"] = smooth_field(rng, (nz, ny, nx + 1), -1.5, 1.5)
    st["v"] = smooth_field(rng, (nz, ny + 1, nx), -0.5, 3.0)
    st["w"] = smooth_field(rng, (nz + 1, ny, nx), -1.5, 1.5)
    st["pressure"] = smooth_field(rng, sh, -0.5, 0.5)
    st["divergence"] = smooth_field(rng, sh, -0.3, 0.3)
    lx, ly, lz = ref.light_dims
    st["scene_light"] = np.stack([smooth_field(rng, (lz, ly, lx), 0, 2.0) for _ in range(3)] +
                                 [smooth_field(rng, (lz, ly, lx), 0, 0.8)], axis=-1)
    st["scene_shadow"] = smooth_field(rng, (lz, ly, lx), 0.2, 1.0)
    st["hdr"] = rng.uniform(0, 1.5, (ref.frame_h, ref.frame_w, 4)).astype(np.float32)
    st["bgra"] = rng.integers(0, 2 ** 32, (ref.frame_h, ref.frame_w), dtype=np.uint64).astype(np.uint32)
    return st


def random_variants(fw, fh):
    base = dict(width=fw, height=fh, cameraYaw=0.25, cameraPitch=0.12, cameraDistance=2.8, raymarchSteps=72,
                emberCount=64)
    v0 = abi.FireSettings(**base, sceneId=0, showGizmos=1)
    v1 = abi.FireSettings(**base, sceneId=1, leftDown=1, mouseX=0.45, mouseY=0.22, wind=0.4, turbulence=1.2,
                          detail=1.1, smoke=1.3, intensity=1.6, showGizmos=1, activeGizmo=0, cinematicMode=1)
    v2 = abi.FireSettings(**base, sceneId=2, rightDown=1, mouseX=0.55, mouseY=0.3, wind=-0.3, emitterRadius=0.3,
                          emitterHeightBandNorm=0.05, burnerCenterCount=2,
                          burnerCenterX=[0.1, -0.3, 0, 0], burnerCenterY=[0.2, 0.1, 0, 0],
                          burnerCenterZ=[-0.1, 0.2, 0, 0], showGizmos=0)
    return [v0, v1, v2]


def case_random(outdir: Path) -> None:
    fw, fh, nx, ny, nz = 48, 32, 17, 21, 11
    ref = refmod.RefFire(abi, fw, fh, nx, ny, nz)
    state = random_state(ref, seed=1234)
    arrays = {f"in/{n}": a for n, a in state.items()}
    meta = {"grid": [nx, ny, nz], "frame": [fw, fh], "light": list(ref.light_dims), "variants": [],
            "time": 1.7}
    for vi, s in enumerate(random_variants(fw, fh)):
        meta["variants"].append(s.as_dict())
        stages = list(STAGE_ORDER)
        for stage in stages:
            for n, a in state.items():
                ref.set(n, a)
            ref.stages(stage, stage, s, 1.7)
            for n in STAGE_OUTPUTS[stage]:
                arrays[f"v{vi}/{stage}/{n}"] = ref.get(n)
            if stage == "metrics":
                sums, bits = ref.last_metrics()
                arrays[f"v{vi}/metrics/sums"] = sums
                arrays[f"v{vi}/metrics/bits"] = bits
        if vi == 0:
            for mode in range(1, 7):
                for n, a in state.items():
                    ref.set(n, a)
                s.renderDebugMode = mode
                ref.stages("render", "render", s, 1.7)
                arrays[f"v0/render_debug{mode}/hdr"] = ref.get("hdr")
            s.renderDebugMode = 0
    save(outdir, "random", arrays, meta)
    ref.close()


def main() -> int:
    outdir = Path(sys.argv[1] if len(sys.argv) > 1 else ROOT / "tests" / "golden")
    outdir.mkdir(parents=True, exist_ok=True)
    case_validation(outdir)
    case_scene(outdir, 1)
    case_scene(outdir, 2)
    case_random(outdir)
    return 0


if __name__ == "__main__":
    sys.exit(main())
