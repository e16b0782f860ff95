"""ctypes binding over libfiresim_b200.so, the sm_100a frame pipeline.

`FireSim` drives the library's singleton scene through the same entry points
a native-firesim caller uses (fireCudaInitialize, fireCudaStepAndRender,
fireCudaStepAndRenderMeasured, the *D3D11 family with a device HDR buffer, ...)
plus the extensions of include/fire_ext.h.  Every call raises FireSimError
with fireCudaLastError() when the library returns false.  There is no CPU
fallback: without the built library or without a CUDA device, construction
fails.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import abi

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libfiresim_b200.so"
# The same library built with FP16 / BF16 storage of the transported fields (FP32 arithmetic).
LIB_PATH_F16 = HERE / "libfiresim_b200_f16.so"
LIB_PATH_BF16 = HERE / "libfiresim_b200_bf16.so"
# The FP32 library built with -DFIRE_BOUNDS_CHECK: guard zones around every
# device buffer, checked by fireCudaCheckGuards (check_guards below).
LIB_PATH_CHECKED = HERE / "libfiresim_b200_checked.so"


class FireSimError(RuntimeError):
    pass


_LIBS: dict = {}


def load_library(precision: str = "f32") -> ctypes.CDLL:
    """Loads the in-tree library (build it with native-firesim_b200/build.py):
    precision "f32" (the reference's storage), "f16" or "bf16" (half storage),
    or "checked" (FP32 storage, the bounds-checking build)."""
    if precision in _LIBS:
        return _LIBS[precision]
    paths = {"f32": LIB_PATH, "f16": LIB_PATH_F16, "bf16": LIB_PATH_BF16, "checked": LIB_PATH_CHECKED}
    if precision not in paths:
        raise FireSimError(f"unknown precision {precision!r}: 'f32', 'f16', 'bf16' or 'checked'")
    path = paths[precision]
    if not path.exists():
        raise FireSimError(f"{path} is missing: run `python native-firesim_b200/build.py` first")
    L = ctypes.CDLL(str(path))
    S = ctypes.POINTER(abi.FireSettings)
    M = ctypes.POINTER(abi.FireCudaFrameMetrics)
    b = ctypes.c_bool
    sig = {
        "fireCudaInitialize": (b, [ctypes.c_int] * 4),
        "fireCudaInitializeGrid": (b, [ctypes.c_int] * 5),
        "fireCudaStepAndRender": (b, [ctypes.c_void_p, S]),
        "fireCudaStepAndRenderMeasured": (b, [ctypes.c_void_p, S, M]),
        "fireCudaSelectDeviceForD3D11": (b, [ctypes.c_void_p]),
        "fireCudaRegisterD3D11Texture": (b, [ctypes.c_void_p]),
        "fireCudaRegisterD3D11TextureSlot": (b, [ctypes.c_int, ctypes.c_void_p]),
        "fireCudaSetD3D11TextureSlot": (b, [ctypes.c_int]),
        "fireCudaStepD3D11": (b, [S]),
        "fireCudaStepAndRenderD3D11": (b, [S]),
        "fireCudaStepAndRenderD3D11Measured": (b, [S, M]),
        "fireCudaRenderD3D11": (b, [S]),
        "fireCudaUnregisterD3D11Texture": (None, []),
        "fireCudaSynchronize": (b, []),
        "fireCudaReset": (b, []),
        "fireCudaGetDiagnostics": (b, [ctypes.POINTER(abi.FireCudaDiagnostics)]),
        "fireCudaShutdown": (None, []),
        "fireCudaLastError": (ctypes.c_char_p, []),
        "fireCudaSelectDevice": (b, [ctypes.c_int]),
        "fireCudaRegisterHdrBufferSlot": (b, [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]),
        "fireCudaSetPressureSolver": (b, [ctypes.c_int, ctypes.c_float]),
        "fireCudaSetPressurePath": (b, [ctypes.c_int]),
        "fireCudaGetPressurePathUsed": (ctypes.c_int, []),
        "fireCudaSetHashLattices": (b, [ctypes.c_int]),
        "fireCudaSetAutotune": (b, [ctypes.c_int]),
        "fireCudaGetTunedBrick": (b, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_float)]),
        "fireCudaSetPressureTolerance": (b, [ctypes.c_double, ctypes.c_int]),
        "fireCudaGetPressureStats": (b, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)]),
        "fireCudaApplySceneContract": (b, [ctypes.c_int, ctypes.c_char_p, S]),
        "fireSceneCreate": (ctypes.c_void_p, [ctypes.c_int] * 6),
        "fireSceneDestroy": (None, [ctypes.c_void_p]),
        "fireSceneDeviceBytes": (ctypes.c_size_t, [ctypes.c_void_p]),
        "fireSceneSetPressureSolver": (b, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]),
        "fireSceneSetHdrBuffer": (b, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]),
        "fireSceneStep": (b, [ctypes.c_void_p, S, ctypes.c_int]),
        "fireSceneSynchronize": (b, [ctypes.c_void_p]),
        "fireSceneGetStream": (b, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
        "fireSceneGetField": (b, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
        "fireBatchStep": (b, [ctypes.POINTER(ctypes.c_void_p), S, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
        "fireServerCreate": (ctypes.c_void_p, [ctypes.c_int, ctypes.c_size_t]),
        "fireServerDestroy": (None, [ctypes.c_void_p]),
        "fireServerSubmit": (b, [ctypes.c_void_p, ctypes.POINTER(abi.FireServeRequest)]),
        "fireServerSetLimits": (b, [ctypes.c_void_p, ctypes.c_longlong]),
        "fireServerSetLatencyTarget": (b, [ctypes.c_void_p, ctypes.c_double]),
        "fireServerRun": (b, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(abi.FireServeReport)]),
        "fireCudaSetResidentSorFault": (b, [ctypes.c_int, ctypes.c_longlong]),
        "fireCudaSetAllocationFault": (b, [ctypes.c_longlong]),
        "fireCudaCheckGuards": (b, [ctypes.POINTER(ctypes.c_int)]),
        "fireCudaPlantGuardByte": (b, [ctypes.c_char_p, ctypes.c_size_t]),
        "fireCudaGetGridInfo": (b, [ctypes.POINTER(ctypes.c_int)]),
        "fireCudaGetField": (b, [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
        "fireCudaSetField": (b, [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
        "fireCudaRunStages": (b, [ctypes.c_int, ctypes.c_int, S, ctypes.c_float]),
        "fireCudaRunStagesAsync": (b, [ctypes.c_int, ctypes.c_int, S, ctypes.c_float]),
        "fireCudaGetTimes": (b, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]),
        "fireCudaSetTimes": (b, [ctypes.c_float, ctypes.c_float, ctypes.c_int]),
        "fireCudaGetStream": (b, [ctypes.POINTER(ctypes.c_void_p)]),
        "fireCudaGetLaunchCount": (b, [ctypes.POINTER(ctypes.c_ulonglong)]),
        "fireCudaBuildInfo": (ctypes.c_char_p, []),
        "fireCudaDefaultPhysicsParams": (None, [ctypes.POINTER(abi.FirePhysicsParams), ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "fireCudaSetPhysicsParams": (b, [ctypes.POINTER(abi.FirePhysicsParams)]),
        "fireCudaGetPhysicsParams": (b, [ctypes.POINTER(abi.FirePhysicsParams)]),
        "fireSceneSetPressureTolerance": (b, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
        "fireSceneSetPhysicsParams": (b, [ctypes.c_void_p, ctypes.POINTER(abi.FirePhysicsParams)]),
        "fireCudaSetPressureMultigrid": (b, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "fireSceneSetPressureMultigrid": (b, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "fireSceneGetPressureStats": (b, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_double)]),
        "fireBatchCreate": (ctypes.c_void_p, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
        "fireBatchDestroy": (None, [ctypes.c_void_p]),
        "fireBatchRun": (b, [ctypes.c_void_p, S, ctypes.POINTER(ctypes.c_int)]),
        "fireBatchSynchronize": (b, [ctypes.c_void_p]),
        "fireBatchGetStream": (b, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
        "fireBatchGetLaunchCount": (b, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[precision] = L
    return L


def last_error(lib=None) -> str:
    return (lib or load_library()).fireCudaLastError().decode()


class FireSim:
    """The library's singleton scene on one GPU."""

    def __init__(self, frame_w: int, frame_h: int, nx: int | None = None, ny: int | None = None,
                 nz: int | None = None, grid_request: tuple[int, int] | None = None, precision: str = "f32"):
        self.lib = load_library(precision)
        self.precision = precision
        if grid_request is not None:
            ok = self.lib.fireCudaInitialize(frame_w, frame_h, grid_request[0], grid_request[1])
        else:
            ok = self.lib.fireCudaInitializeGrid(frame_w, frame_h, nx, ny, nz)
        self._check(ok, "initialize")
        dims = (ctypes.c_int * 8)()
        self._check(self.lib.fireCudaGetGridInfo(dims), "grid info")
        self.nx, self.ny, self.nz, lx, ly, lz, self.frame_w, self.frame_h = list(dims)
        self.light_dims = (lx, ly, lz)

    def _check(self, ok, what):
        if not ok:
            raise FireSimError(f"{what}: {last_error(self.lib)}")

    def close(self):
        self.lib.fireCudaShutdown()

    # --- the reference's entry points -------------------------------------
    def step_and_render(self, settings, metrics: bool = False):
        """fireCudaStepAndRender(Measured): returns (bgra HxW uint32, metrics or None)."""
        bgra = np.zeros((self.frame_h, self.frame_w), dtype=np.uint32)
        if metrics:
            m = abi.FireCudaFrameMetrics()
            self._check(self.lib.fireCudaStepAndRenderMeasured(bgra.ctypes.data, ctypes.byref(settings), ctypes.byref(m)),
                        "fireCudaStepAndRenderMeasured")
            return bgra, m
        self._check(self.lib.fireCudaStepAndRender(bgra.ctypes.data, ctypes.byref(settings)), "fireCudaStepAndRender")
        return bgra, None

    def step(self, settings):
        self._check(self.lib.fireCudaStepD3D11(ctypes.byref(settings)), "fireCudaStepD3D11")

    def step_and_render_hdr(self, settings, metrics: bool = False):
        if metrics:
            m = abi.FireCudaFrameMetrics()
            self._check(self.lib.fireCudaStepAndRenderD3D11Measured(ctypes.byref(settings), ctypes.byref(m)),
                        "fireCudaStepAndRenderD3D11Measured")
            return m
        self._check(self.lib.fireCudaStepAndRenderD3D11(ctypes.byref(settings)), "fireCudaStepAndRenderD3D11")
        return None

    def render_hdr(self, settings):
        self._check(self.lib.fireCudaRenderD3D11(ctypes.byref(settings)), "fireCudaRenderD3D11")

    def register_hdr_slot(self, slot: int, device_ptr: int, pitch_bytes: int, fmt: int = 0):
        self._check(self.lib.fireCudaRegisterHdrBufferSlot(slot, ctypes.c_void_p(device_ptr), pitch_bytes, fmt),
                    "fireCudaRegisterHdrBufferSlot")

    def set_hdr_slot(self, slot: int):
        self._check(self.lib.fireCudaSetD3D11TextureSlot(slot), "fireCudaSetD3D11TextureSlot")

    def synchronize(self):
        self._check(self.lib.fireCudaSynchronize(), "fireCudaSynchronize")

    def reset(self):
        self._check(self.lib.fireCudaReset(), "fireCudaReset")

    def diagnostics(self) -> abi.FireCudaDiagnostics:
        d = abi.FireCudaDiagnostics()
        self._check(self.lib.fireCudaGetDiagnostics(ctypes.byref(d)), "fireCudaGetDiagnostics")
        return d

    # --- extensions ---------------------------------------------------------
    def set_pressure_solver(self, iterations: int, omega: float):
        self._check(self.lib.fireCudaSetPressureSolver(iterations, omega), "fireCudaSetPressureSolver")

    def set_pressure_path(self, path: int):
        """0 automatic, 1 colour-split (one launch per half sweep, as a graph), 2 shared-memory-resident."""
        self._check(self.lib.fireCudaSetPressurePath(path), "fireCudaSetPressurePath")

    def set_resident_sor_fault(self, silent_brick: int = -1, wait_us: int = 1_000_000):
        """Fault injection for the resident SOR's bounded neighbour waits."""
        self._check(self.lib.fireCudaSetResidentSorFault(silent_brick, wait_us), "fireCudaSetResidentSorFault")

    def set_pressure_tolerance(self, max_residual: float, check_every: int = 10):
        """Residual-gated SOR: stop once max |r| <= max_residual (0 = fixed iteration count)."""
        self._check(self.lib.fireCudaSetPressureTolerance(max_residual, check_every), "fireCudaSetPressureTolerance")

    def pressure_stats(self):
        """(iterations, max |r|, L2 residual) of the latest gated solve."""
        it, mr, l2 = ctypes.c_int(), ctypes.c_float(), ctypes.c_double()
        self._check(self.lib.fireCudaGetPressureStats(ctypes.byref(it), ctypes.byref(mr), ctypes.byref(l2)), "fireCudaGetPressureStats")
        return it.value, mr.value, l2.value

    def set_physics(self, params) -> None:
        """FirePhysicsParams for the following passes (mode 1: config physics)."""
        self._check(self.lib.fireCudaSetPhysicsParams(ctypes.byref(params)), "fireCudaSetPhysicsParams")

    def set_pressure_multigrid(self, max_cycles: int, pre_smooth: int = 2, post_smooth: int = 2) -> None:
        """Multigrid V-cycles for the config physics with a Dirichlet top (0 cycles: red-black SOR)."""
        self._check(self.lib.fireCudaSetPressureMultigrid(max_cycles, pre_smooth, post_smooth), "fireCudaSetPressureMultigrid")

    def physics(self):
        p = abi.FirePhysicsParams()
        self._check(self.lib.fireCudaGetPhysicsParams(ctypes.byref(p)), "fireCudaGetPhysicsParams")
        return p

    def set_hash_lattices(self, enabled: bool):
        """Hash-lattice tables for the fbm fields on (default) or off (in-place hashing, same bits)."""
        self._check(self.lib.fireCudaSetHashLattices(1 if enabled else 0), "fireCudaSetHashLattices")

    def pressure_path_used(self) -> int:
        """Path of the latest pressure solve: 0 none yet, 1 colour-split SOR, 2 resident SOR, 3 multigrid."""
        return int(self.lib.fireCudaGetPressurePathUsed())

    def shape_of(self, name: str):
        nx, ny, nz = self.nx, self.ny, self.nz
        lx, ly, lz = self.light_dims
        return {
            "u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx),
            "scene_light": (lz, ly, lx, 4), "scene_shadow": (lz, ly, lx),
            "hdr": (self.frame_h, self.frame_w, 4), "bgra": (self.frame_h, self.frame_w),
            "config_transmittance": ((nz + 1) // 2, (ny + 1) // 2, (nx + 1) // 2),
        }.get(name, (nz, ny, nx))

    def get(self, name: str) -> np.ndarray:
        dtype = np.uint32 if name == "bgra" else np.float32
        out = np.empty(self.shape_of(name), dtype=dtype)
        self._check(self.lib.fireCudaGetField(abi.FIELDS[name], out.ctypes.data, out.nbytes), f"get {name}")
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        dtype = np.uint32 if name == "bgra" else np.float32
        a = np.ascontiguousarray(arr, dtype=dtype).reshape(self.shape_of(name))
        self._check(self.lib.fireCudaSetField(abi.FIELDS[name], a.ctypes.data, a.nbytes), f"set {name}")

    def stages(self, first: str, last: str, settings, time: float, wait: bool = True) -> None:
        """Runs stages first..last; with wait=False only queues them on stream()."""
        s = abi.STAGES
        fn = self.lib.fireCudaRunStages if wait else self.lib.fireCudaRunStagesAsync
        self._check(fn(s[first], s[last], ctypes.byref(settings), time), f"stages {first}..{last}")

    def times(self):
        t, r, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        self._check(self.lib.fireCudaGetTimes(ctypes.byref(t), ctypes.byref(r), ctypes.byref(f)), "times")
        return t.value, r.value, f.value

    def stream(self) -> int:
        """cudaStream_t of the scene, as an integer handle."""
        ptr = ctypes.c_void_p()
        self._check(self.lib.fireCudaGetStream(ctypes.byref(ptr)), "fireCudaGetStream")
        return int(ptr.value or 0)

    def launch_count(self) -> int:
        n = ctypes.c_ulonglong()
        self._check(self.lib.fireCudaGetLaunchCount(ctypes.byref(n)), "fireCudaGetLaunchCount")
        return int(n.value)

    def set_times(self, sim_time: float, render_time: float, frame_index: int) -> None:
        self._check(self.lib.fireCudaSetTimes(sim_time, render_time, frame_index), "set times")


def set_autotune(enabled: bool, precision: str = "f32") -> None:
    """The resident SOR's brick-shape autotuner on (default) or off, process-wide."""
    lib = load_library(precision)
    if not lib.fireCudaSetAutotune(1 if enabled else 0):
        raise FireSimError(f"fireCudaSetAutotune: {last_error(lib)}")


def check_guards(precision: str = "checked") -> int:
    """Scans the guard zones of the bounds-checking build's device buffers
    (fireCudaCheckGuards): returns 0 when every zone is intact, raises
    FireSimError naming the first changed buffer otherwise, and returns -1
    for a library built without the checks."""
    lib = load_library(precision)
    n = ctypes.c_int(-1)
    if lib.fireCudaCheckGuards(ctypes.byref(n)):
        return 0
    if n.value < 0:
        return -1
    raise FireSimError(lib.fireCudaLastError().decode())


def tuned_brick(nx: int, ny: int, nz: int, precision: str = "f32"):
    """(brick x, ms per solve with 32x16x16 bricks, with 16x16x16) as the autotuner
    measured them for this grid on the current device, or None if not timed."""
    lib = load_library(precision)
    bx, a, c = ctypes.c_int(), ctypes.c_float(), ctypes.c_float()
    if not lib.fireCudaGetTunedBrick(nx, ny, nz, ctypes.byref(bx), ctypes.byref(a), ctypes.byref(c)):
        return None
    return bx.value, a.value, c.value


def apply_scene_contract(scene_id: int, fire_scenes_dir, settings) -> None:
    """Fills the emitter fields of `settings` from the scene's contract files
    (fireCudaApplySceneContract); None gives the built-in values."""
    lib = load_library()
    path = None if fire_scenes_dir is None else str(fire_scenes_dir).encode()
    if not lib.fireCudaApplySceneContract(scene_id, path, ctypes.byref(settings)):
        raise FireSimError(f"fireCudaApplySceneContract: {last_error()}")


class Scene:
    """A FireScene handle (fireSceneCreate ...): an independent scene with its
    own fields and stream; many of them run side by side on one GPU."""

    def __init__(self, frame_w: int, frame_h: int, nx: int, ny: int, nz: int, device: int = 0, precision: str = "f32"):
        self.lib = load_library(precision)
        self.h = self.lib.fireSceneCreate(device, frame_w, frame_h, nx, ny, nz)
        if not self.h:
            raise FireSimError(f"fireSceneCreate: {last_error(self.lib)}")
        self.nx, self.ny, self.nz, self.frame_w, self.frame_h = nx, ny, nz, frame_w, frame_h

    def _check(self, ok, what):
        if not ok:
            raise FireSimError(f"{what}: {last_error(self.lib)}")

    def close(self):
        if self.h:
            self.lib.fireSceneDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass

    def device_bytes(self) -> int:
        return int(self.lib.fireSceneDeviceBytes(self.h))

    def set_pressure_solver(self, iterations: int, omega: float):
        self._check(self.lib.fireSceneSetPressureSolver(self.h, iterations, omega), "fireSceneSetPressureSolver")

    def set_pressure_tolerance(self, max_residual: float, check_every: int = 10):
        self._check(self.lib.fireSceneSetPressureTolerance(self.h, max_residual, check_every), "fireSceneSetPressureTolerance")

    def set_physics(self, params) -> None:
        self._check(self.lib.fireSceneSetPhysicsParams(self.h, ctypes.byref(params)), "fireSceneSetPhysicsParams")

    def set_pressure_multigrid(self, max_cycles: int, pre_smooth: int = 2, post_smooth: int = 2) -> None:
        self._check(self.lib.fireSceneSetPressureMultigrid(self.h, max_cycles, pre_smooth, post_smooth),
                    "fireSceneSetPressureMultigrid")

    def set_hdr_buffer(self, device_ptr: int, pitch_bytes: int, fmt: int = 0):
        self._check(self.lib.fireSceneSetHdrBuffer(self.h, device_ptr, pitch_bytes, fmt), "fireSceneSetHdrBuffer")

    def step(self, settings, render: bool = False):
        self._check(self.lib.fireSceneStep(self.h, ctypes.byref(settings), 1 if render else 0), "fireSceneStep")

    def synchronize(self):
        self._check(self.lib.fireSceneSynchronize(self.h), "fireSceneSynchronize")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.fireSceneGetStream(self.h, ctypes.byref(s)), "fireSceneGetStream")
        return s.value or 0

    def get(self, name: str) -> np.ndarray:
        shape = {"u": (self.nz, self.ny, self.nx + 1), "v": (self.nz, self.ny + 1, self.nx),
                 "w": (self.nz + 1, self.ny, self.nx), "hdr": (self.frame_h, self.frame_w, 4)}.get(name, (self.nz, self.ny, self.nx))
        out = np.empty(shape, dtype=np.float32)
        self._check(self.lib.fireSceneGetField(self.h, abi.FIELDS[name], out.ctypes.data, out.nbytes), f"get {name}")
        return out

    def pressure_stats(self):
        """(iterations or multigrid cycles, max |r|, L2 residual) of the latest gated solve."""
        it, m, l2 = ctypes.c_int(), ctypes.c_float(), ctypes.c_double()
        self._check(self.lib.fireSceneGetPressureStats(self.h, ctypes.byref(it), ctypes.byref(m), ctypes.byref(l2)),
                    "fireSceneGetPressureStats")
        return it.value, m.value, l2.value


class Batch:
    """fireBatch*: scenes of the config physics (p = 0 on the top face, multigrid
    solve) stepped together, one launch per stage over all of them."""

    def __init__(self, scenes):
        self.scenes = list(scenes)
        self.lib = self.scenes[0].lib
        handles = (ctypes.c_void_p * len(self.scenes))(*[s.h for s in self.scenes])
        self.h = self.lib.fireBatchCreate(handles, len(self.scenes))
        if not self.h:
            raise FireSimError(f"fireBatchCreate: {last_error(self.lib)}")

    def run(self, settings, render=None) -> None:
        n = len(self.scenes)
        arr = (abi.FireSettings * n)(*settings)
        flags = None if render is None else (ctypes.c_int * n)(*[1 if r else 0 for r in render])
        if not self.lib.fireBatchRun(self.h, arr, flags):
            raise FireSimError(f"fireBatchRun: {last_error(self.lib)}")

    def synchronize(self) -> None:
        if not self.lib.fireBatchSynchronize(self.h):
            raise FireSimError(f"fireBatchSynchronize: {last_error(self.lib)}")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        if not self.lib.fireBatchGetStream(self.h, ctypes.byref(s)):
            raise FireSimError(f"fireBatchGetStream: {last_error(self.lib)}")
        return s.value or 0

    def launch_count(self) -> int:
        c = ctypes.c_ulonglong()
        if not self.lib.fireBatchGetLaunchCount(self.h, ctypes.byref(c)):
            raise FireSimError(f"fireBatchGetLaunchCount: {last_error(self.lib)}")
        return int(c.value)

    def close(self) -> None:
        if self.h:
            self.lib.fireBatchDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


def batch_step(scenes, settings, render=None) -> None:
    """fireBatchStep: one queued step of every scene (settings[i] for scenes[i])."""
    lib = scenes[0].lib if scenes else load_library()
    n = len(scenes)
    handles = (ctypes.c_void_p * n)(*[s.h for s in scenes])
    arr = (abi.FireSettings * n)(*settings)
    flags = None if render is None else (ctypes.c_int * n)(*[1 if r else 0 for r in render])
    if not lib.fireBatchStep(handles, arr, flags, n):
        raise FireSimError(f"fireBatchStep: {last_error(lib)}")


class Server:
    """fireServer*: requests arrive over time, are admitted within a device-memory
    budget and all admitted scenes advance one step per round."""

    def __init__(self, budget_bytes: int, device: int = 0, precision: str = "f32"):
        self.lib = load_library(precision)
        self.h = self.lib.fireServerCreate(device, budget_bytes)
        if not self.h:
            raise FireSimError(f"fireServerCreate: {last_error(self.lib)}")

    def set_limits(self, max_active_voxels: int) -> None:
        """Admit only while the admitted scenes hold at most this many cells (0 = no limit)."""
        if not self.lib.fireServerSetLimits(self.h, max_active_voxels):
            raise FireSimError(f"fireServerSetLimits: {last_error(self.lib)}")

    def set_latency_target(self, round_ms: float) -> None:
        """Batched loop: admit while the predicted round time stays within round_ms (0 = off)."""
        if not self.lib.fireServerSetLatencyTarget(self.h, round_ms):
            raise FireSimError(f"fireServerSetLatencyTarget: {last_error(self.lib)}")

    def submit(self, request) -> None:
        if not self.lib.fireServerSubmit(self.h, ctypes.byref(request)):
            raise FireSimError(f"fireServerSubmit: {last_error(self.lib)}")

    def run(self, max_seconds: float) -> dict:
        rep = abi.FireServeReport()
        if not self.lib.fireServerRun(self.h, max_seconds, ctypes.byref(rep)):
            raise FireSimError(f"fireServerRun: {last_error(self.lib)}")
        return rep.as_dict()

    def close(self):
        if self.h:
            self.lib.fireServerDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
