"""ctypes mirror of the reference ABI structs (include/fire_cuda.h).

Field order, types and defaults follow src/fire_cuda.h:5-100 of native-firesim,
so a FireSettings built here has the byte layout the reference's callers pass.
"""
from __future__ import annotations

import ctypes

# Field ids shared by every copy/compare entry point (FIRE_FIELD_* in include/fire_ext.h).
FIELDS = {
    "heat": 0, "fuel": 1, "oxygen": 2, "soot": 3, "char": 4, "ash": 5, "pyrolysis": 6,
    "progress": 7, "turbulence_energy": 8, "soot_optics": 9, "pressure": 10, "divergence": 11,
    "u": 12, "v": 13, "w": 14, "scene_light": 15, "scene_shadow": 16, "hdr": 17, "bgra": 18,
    "divergence_after": 19, "config_transmittance": 20,
}
SCALAR_FIELDS = ["heat", "fuel", "oxygen", "soot", "char", "ash", "pyrolysis", "progress",
                 "turbulence_energy", "soot_optics"]

# Stage ids (FIRE_STAGE_* in include/fire_ext.h), in step order.
STAGES = {
    "advect_velocity": 0, "advect_react": 1, "force": 2, "velocity_boundary": 3, "divergence": 4,
    "pressure_sor": 5, "subtract": 6, "wall_boundary": 7, "light_build": 8, "light_propagate": 9,
    "render": 10, "embers": 11, "tonemap": 12, "overlay": 13, "metrics": 14, "reset": 15,
}


class FireCudaDiagnostics(ctypes.Structure):
    _fields_ = [
        ("driverVersion", ctypes.c_int), ("runtimeVersion", ctypes.c_int), ("deviceCount", ctypes.c_int),
        ("activeDevice", ctypes.c_int), ("computeMajor", ctypes.c_int), ("computeMinor", ctypes.c_int),
        ("totalGlobalMem", ctypes.c_uint64), ("deviceName", ctypes.c_char * 128),
    ]

    def __init__(self):
        super().__init__()
        self.activeDevice = -1


_METRIC_INTS = ["frameIndex", "gridX", "gridY", "gridZ", "pressureIterations", "invalidCells"]
_METRIC_FLOATS = [
    "timeSeconds", "gpuSolveMs", "gpuRenderMs", "gpuVelocityMs", "gpuReactionMs", "gpuProjectionMs",
    "gpuLightingMs", "gpuRaymarchMs", "gpuPackMs", "heatSum", "fuelSum", "oxygenSum", "sootSum", "charSum",
    "ashSum", "pyrolysisSum", "progressSum", "turbulenceEnergySum", "sootOpticalDepthSum", "maxHeat",
    "maxFuel", "maxSoot", "maxPyrolysis", "maxProgress", "maxTurbulenceEnergy", "flameHeightMeters",
    "meanOpticalDepth", "meanSceneLight", "meanSceneShadow", "flameMassProxy", "smokeMassProxy",
    "flameSmokeOverlapProxy", "meanVolumetricShadow", "meanRoomIrradiance", "heatReleaseProxy",
    "divergenceBeforeL2", "divergenceBeforeMax", "divergenceAfterL2", "divergenceAfterMax",
    "divergenceReduction",
]


class FireCudaFrameMetrics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in _METRIC_INTS] + [(n, ctypes.c_float) for n in _METRIC_FLOATS]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class FireSettings(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("dt", ctypes.c_float),
        ("mouseX", ctypes.c_float), ("mouseY", ctypes.c_float), ("leftDown", ctypes.c_int),
        ("rightDown", ctypes.c_int), ("reset", ctypes.c_int), ("showGizmos", ctypes.c_int),
        ("activeGizmo", ctypes.c_int), ("sceneId", ctypes.c_int), ("wind", ctypes.c_float),
        ("turbulence", ctypes.c_float), ("detail", ctypes.c_float), ("smoke", ctypes.c_float),
        ("intensity", ctypes.c_float), ("cameraYaw", ctypes.c_float), ("cameraPitch", ctypes.c_float),
        ("cameraDistance", ctypes.c_float), ("cinematicMode", ctypes.c_int), ("raymarchSteps", ctypes.c_int),
        ("emberCount", ctypes.c_int), ("renderDebugMode", ctypes.c_int), ("exposure", ctypes.c_float),
        ("reflectionGain", ctypes.c_float), ("smokeDarkness", ctypes.c_float),
        ("emitterCenterX", ctypes.c_float), ("emitterCenterZ", ctypes.c_float),
        ("emitterHeightNorm", ctypes.c_float), ("emitterHeightBandNorm", ctypes.c_float),
        ("emitterRadius", ctypes.c_float), ("burnerCenterCount", ctypes.c_int),
        ("burnerCenterX", ctypes.c_float * 4), ("burnerCenterY", ctypes.c_float * 4),
        ("burnerCenterZ", ctypes.c_float * 4),
    ]

    # src/fire_cuda.h:64-100 defaults.
    _DEFAULTS = dict(
        width=1280, height=720, dt=1.0 / 60.0, mouseX=0.5, mouseY=0.12, leftDown=0, rightDown=0, reset=0,
        showGizmos=1, activeGizmo=1, sceneId=0, wind=0.0, turbulence=0.72, detail=0.88, smoke=0.92,
        intensity=1.0, cameraYaw=0.0, cameraPitch=0.18, cameraDistance=3.35, cinematicMode=0,
        raymarchSteps=56, emberCount=96, renderDebugMode=0, exposure=1.0, reflectionGain=1.0,
        smokeDarkness=1.0, emitterCenterX=0.0, emitterCenterZ=0.0, emitterHeightNorm=0.0,
        emitterHeightBandNorm=0.06, emitterRadius=0.48, burnerCenterCount=0,
    )

    def __init__(self, **kw):
        super().__init__()
        for k, v in {**self._DEFAULTS, **kw}.items():
            if k.startswith("burnerCenter") and k != "burnerCenterCount":
                arr = getattr(self, k)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(self, k, v)

    def as_dict(self) -> dict:
        out = {}
        for n, _ in self._fields_:
            v = getattr(self, n)
            out[n] = list(v) if n.startswith("burnerCenter") and n != "burnerCenterCount" else v
        return out


def f32(x: float) -> float:
    """Round a Python float to the nearest binary32 value."""
    return ctypes.c_float(x).value


# Canonical host constants, src/main.cpp:33-43, applied by applyCanonicalFireSettings (src/main.cpp:2758-2770).
CANONICAL = dict(cinematicMode=1, raymarchSteps=104, emberCount=176, exposure=0.84, reflectionGain=0.54,
                 smokeDarkness=1.26, intensity=1.42, smoke=0.96, turbulence=1.34, renderDebugMode=0)


def validation_settings(frame: int, scene: int = 0, width: int = 960, height: int = 540,
                        pool_fire: bool = False, fire_scenes_dir=None) -> FireSettings:
    """FireSettings of frame `frame` of the reference's validation harness.

    Restates src/main.cpp:4284-4311 (runValidation): deterministic mouse/wind
    motion, canonical constants, then the validation floors for turbulence,
    smoke and intensity and the fixed validation camera.  Scene emitter
    parameters are the built-in defaults of SceneEmitterParams
    (src/main.cpp:173, used when no scene contract is loaded); with
    `fire_scenes_dir` they come from the scene's contract files, applied at the
    same point as the reference's applySceneEmitterParams (:4305), through
    fireCudaApplySceneContract.
    """
    import numpy as np
    f = np.float32
    s = FireSettings(width=width, height=height, dt=1.0 / 60.0)
    if pool_fire:
        s.mouseX, s.mouseY = 0.50, 0.12
    else:
        s.mouseX = float(f(0.50) + f(0.07) * np.sin(f(frame) * f(0.071)))
        s.mouseY = float(f(0.12) + f(0.035) * np.sin(f(frame) * f(0.053)))
    s.leftDown = 0
    s.rightDown = 0
    s.showGizmos = 0
    s.activeGizmo = 1
    s.sceneId = scene
    s.reset = 1 if frame == 0 else 0
    s.wind = 0.0 if pool_fire else float(f(0.10) + f(0.05) * np.sin(f(frame) * f(0.037)))
    s.detail = 0.98
    for k, v in CANONICAL.items():
        setattr(s, k, v)
    if fire_scenes_dir is not None:
        from . import firesim  # noqa: PLC0415
        firesim.apply_scene_contract(scene, fire_scenes_dir, s)
    s.turbulence = max(s.turbulence, f32(1.08))
    s.smoke = max(s.smoke, f32(1.02))
    s.intensity = max(s.intensity, f32(1.18))
    s.cameraYaw = 0.18
    s.cameraPitch = 0.08
    s.cameraDistance = 2.62
    return s


# ---- Config physics (FirePhysicsParams.mode 1, include/fire_ext.h) ----------

MAX_EMITTERS = 4


class FireEmitterDisk(ctypes.Structure):
    """include/fire_ext.h FireEmitterDisk."""
    _fields_ = [
        ("centerX", ctypes.c_float), ("centerY", ctypes.c_float), ("centerZ", ctypes.c_float),
        ("radius", ctypes.c_float), ("fuel", ctypes.c_float), ("heat", ctypes.c_float),
        ("upVelocity", ctypes.c_float), ("jitterScale", ctypes.c_float), ("seed", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


_PHYSICS_FLOATS_A = ["dt", "buoyancyHeat", "buoyancySoot", "ambientHeat", "burnRate", "ignitionHeat",
                     "heatRelease", "sootYield", "cooling", "sootDecay", "vorticityEps", "windX", "windZ",
                     "noiseAmplitude", "noisePeriod"]
_PHYSICS_FLOATS_B = ["lightX", "lightY", "lightZ", "lightIntensity", "extinction", "fuelExtinction",
                     "emission", "albedo", "eyeX", "eyeY", "eyeZ", "targetX", "targetY", "targetZ", "fovYDegrees"]


class FirePhysicsParams(ctypes.Structure):
    """include/fire_ext.h FirePhysicsParams (fill it with default_physics first)."""
    _fields_ = ([("mode", ctypes.c_int)] + [(n, ctypes.c_float) for n in _PHYSICS_FLOATS_A] +
                [("noiseSeed", ctypes.c_uint32), ("emitterCount", ctypes.c_int),
                 ("emitters", FireEmitterDisk * MAX_EMITTERS), ("primarySamples", ctypes.c_int),
                 ("lightSamples", ctypes.c_int)] + [(n, ctypes.c_float) for n in _PHYSICS_FLOATS_B] +
                [("pressureTop", ctypes.c_int)])

    def as_dict(self) -> dict:
        out = {n: getattr(self, n) for n, _ in self._fields_ if n != "emitters"}
        out["emitters"] = [{k: getattr(self.emitters[e], k) for k, _ in FireEmitterDisk._fields_}
                           for e in range(self.emitterCount)]
        return out


class FireServeRequest(ctypes.Structure):
    """include/fire_ext.h FireServeRequest."""
    _fields_ = [
        ("id", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("frameW", ctypes.c_int), ("frameH", ctypes.c_int), ("steps", ctypes.c_int), ("renderEvery", ctypes.c_int),
        ("sorIterations", ctypes.c_int), ("sorOmega", ctypes.c_float), ("arrivalSeconds", ctypes.c_double),
        ("settings", FireSettings), ("resultHeat", ctypes.c_void_p), ("resultHdr", ctypes.c_void_p),
        ("physics", FirePhysicsParams), ("multigridCycles", ctypes.c_int), ("multigridPre", ctypes.c_int),
        ("multigridPost", ctypes.c_int), ("pressureTolerance", ctypes.c_double),
    ]


class FireServeReport(ctypes.Structure):
    """include/fire_ext.h FireServeReport."""
    _fields_ = [
        ("submitted", ctypes.c_int), ("completed", ctypes.c_int), ("admittedPeak", ctypes.c_int),
        ("seconds", ctypes.c_double), ("voxelSteps", ctypes.c_double),
        ("stepMsP50", ctypes.c_double), ("stepMsP95", ctypes.c_double), ("stepMsP99", ctypes.c_double),
        ("stepMsMax", ctypes.c_double), ("frameMsP50", ctypes.c_double), ("frameMsP95", ctypes.c_double),
        ("frameMsP99", ctypes.c_double), ("queueMsP50", ctypes.c_double), ("queueMsP99", ctypes.c_double),
        ("deviceBytesPeak", ctypes.c_size_t),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_physics(nx: int, ny: int, nz: int, lib=None) -> FirePhysicsParams:
    """fireCudaDefaultPhysicsParams (host only, needs no GPU)."""
    if lib is None:
        from . import firesim  # noqa: PLC0415
        lib = firesim.load_library()
    p = FirePhysicsParams()
    lib.fireCudaDefaultPhysicsParams(ctypes.byref(p), nx, ny, nz)
    return p


def _disk(cx, cy, cz, r, seed, fuel=1.0, heat=1.0, up=2.0, jitter=0.2) -> FireEmitterDisk:
    return FireEmitterDisk(centerX=cx, centerY=cy, centerZ=cz, radius=r, fuel=fuel, heat=heat, upVelocity=up,
                           jitterScale=jitter, seed=seed)


def _config_constants(p: FirePhysicsParams) -> FirePhysicsParams:
    """The physics constants shared by every config workload."""
    p.mode = 1
    p.dt = 1.0 / 60.0
    p.buoyancyHeat, p.buoyancySoot = 1.0, 0.1
    p.burnRate, p.sootYield = 0.5, 0.3
    p.vorticityEps = 0.3
    return p


def config_scene(nx: int, ny: int, nz: int, center_x: float, center_z: float, radius: float, wind_x: float,
                 wind_z: float, seed: int, lib=None) -> FirePhysicsParams:
    """One scene of the batched and served config workloads: the shared
    constants, one disk emitter on row 2 (F = T = 1, upward 2 cells/step,
    jitter 0.2 from `seed`), wind (wind_x, wind_z), 64 primary and 32 light
    samples, the light above the grid's centre."""
    p = _config_constants(default_physics(nx, ny, nz, lib))
    p.emitterCount = 1
    p.emitters[0] = _disk(center_x, 2, center_z, radius, seed)
    p.windX, p.windZ = wind_x, wind_z
    p.primarySamples, p.lightSamples = 64, 32
    return p


def config_workload(name: str, lib=None) -> dict:
    """The three single-scene workloads of the config physics, as FirePhysicsParams
    plus the solver, render and run settings they are stated with.

    c1: 64^3, disk emitter r 6 at (32, 4, 32), F = T = 1 with jitter 0.2 from
        seed 1, upward 2 cells/step; dt 1/60, confinement 0.3, buoyancy 0.1
        (soot) and 1.0 (heat), burn 0.5/s, soot yield 0.3; SOR 40 at omega 1.7;
        100 steps; one 256^2 frame, 64 samples, 32 light samples, point light
        at (32, 90, 32).
    c2: 128^3, the same physics with the emitter scaled x2 (r 12 at (64, 8,
        64)), wind 0.5 on x, curl of value noise (seed 7, amplitude 0.4, period
        16); SOR 60 at omega 1.8; 200 steps; a 512^2 frame every 10 steps, 128
        samples, 48 light samples, light at (64, 180, 64).
    c3: 256^3, BF16 storage; emitters r 16 at (96, 6, 128) and r 10 at (170,
        6, 110), seed 3; SOR until max |r| <= 1e-5 or 120 iterations at omega
        1.85; 100 steps.
    """
    sizes = {"c1": 64, "c2": 128, "c3": 256}
    if name not in sizes:
        raise ValueError(f"unknown config workload {name!r}: c1, c2 or c3")
    n = sizes[name]
    p = _config_constants(default_physics(n, n, n, lib))
    w = dict(name=name, grid=(n, n, n), physics=p, tolerance=0.0, check_every=10, precision="f32")
    if name == "c1":
        p.emitterCount = 1
        p.emitters[0] = _disk(32, 4, 32, 6, 1)
        p.primarySamples, p.lightSamples = 64, 32
        p.lightX, p.lightY, p.lightZ = 32, 90, 32
        w.update(frame=(256, 256), sor=(40, 1.7), steps=100, render_every=100)
    elif name == "c2":
        p.emitterCount = 1
        p.emitters[0] = _disk(64, 8, 64, 12, 1)
        p.windX = 0.5
        p.noiseSeed, p.noiseAmplitude, p.noisePeriod = 7, 0.4, 16.0
        p.primarySamples, p.lightSamples = 128, 48
        p.lightX, p.lightY, p.lightZ = 64, 180, 64
        w.update(frame=(512, 512), sor=(60, 1.8), steps=200, render_every=10)
    else:
        p.emitterCount = 2
        p.emitters[0] = _disk(96, 6, 128, 16, 3)
        p.emitters[1] = _disk(170, 6, 110, 10, 3)
        p.primarySamples, p.lightSamples = 128, 48
        p.lightX, p.lightY, p.lightZ = 128, 360, 128
        w.update(frame=(512, 512), sor=(120, 1.85), tolerance=1e-5, steps=100, render_every=100, precision="bf16")
    return w
