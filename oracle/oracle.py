"""ctypes binding for the CPU oracle (oracle/_build/libfire_oracle.so).

TEST INFRASTRUCTURE, NOT PRODUCT CODE: only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg use it.  The interface mirrors oracle/ref.py
(the reference's own CUDA code) so a test can run the same script on either.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load_library():
    import build_oracle  # noqa: PLC0415  (oracle/ is on sys.path for its users)
    lib = ctypes.CDLL(str(build_oracle.build()))
    return lib


_LIB = None


def lib(abi):
    global _LIB
    if _LIB is None:
        L = load_library()
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_int] * 6
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_light_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.oracle_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.oracle_get_field_f64.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.oracle_stages.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(abi.FireSettings),
                                    ctypes.c_float]
        L.oracle_set_pressure_solver.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(abi.FireSettings),
                                  ctypes.POINTER(abi.FireCudaFrameMetrics), ctypes.c_int]
        L.oracle_last_metrics.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        L.oracle_times.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                   ctypes.POINTER(ctypes.c_int)]
        L.oracle_set_times.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


class OracleFire:
    """One scene on the CPU. precision: 'f32' (the reference's arithmetic) or 'f64'."""

    def __init__(self, abi, frame_w: int, frame_h: int, nx: int, ny: int, nz: int, precision: str = "f32"):
        self.abi = abi
        self.lib = lib(abi)
        self.precision = precision
        self.h = self.lib.oracle_create(0 if precision == "f32" else 1, frame_w, frame_h, nx, ny, nz)
        if not self.h:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        self.frame_w, self.frame_h = frame_w, frame_h
        self.nx, self.ny, self.nz = nx, ny, nz
        dims = (ctypes.c_int * 3)()
        self.lib.oracle_light_dims(self.h, dims)
        self.light_dims = tuple(dims)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.oracle_destroy(h)
            self.h = None

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {self.lib.oracle_last_error().decode()}")

    def shape_of(self, name: str):
        nx, ny, nz = self.nx, self.ny, self.nz
        lx, ly, lz = self.light_dims
        return {
            "u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx),
            "scene_light": (lz, ly, lx, 4), "scene_shadow": (lz, ly, lx),
            "hdr": (self.frame_h, self.frame_w, 4), "bgra": (self.frame_h, self.frame_w),
        }.get(name, (nz, ny, nx))

    def get(self, name: str) -> np.ndarray:
        dtype = np.uint32 if name == "bgra" else np.float32
        out = np.empty(self.shape_of(name), dtype=dtype)
        self._check(self.lib.oracle_get_field(self.h, self.abi.FIELDS[name], out.ctypes.data, out.nbytes), f"get {name}")
        return out

    def get64(self, name: str) -> np.ndarray:
        out = np.empty(self.shape_of(name), dtype=np.float64)
        self._check(self.lib.oracle_get_field_f64(self.h, self.abi.FIELDS[name], out.ctypes.data, out.size),
                    f"get64 {name}")
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        dtype = np.uint32 if name == "bgra" else np.float32
        a = np.ascontiguousarray(arr, dtype=dtype).reshape(self.shape_of(name))
        self._check(self.lib.oracle_set_field(self.h, self.abi.FIELDS[name], a.ctypes.data, a.nbytes), f"set {name}")

    def stages(self, first: str, last: str, settings, time: float) -> None:
        s = self.abi.STAGES
        self._check(self.lib.oracle_stages(self.h, s[first], s[last], ctypes.byref(settings), time),
                    f"stages {first}..{last}")

    def set_pressure_solver(self, iterations: int, omega: float) -> None:
        self.lib.oracle_set_pressure_solver(self.h, iterations, omega)

    def step(self, settings, mode: int = 1):
        bgra = np.zeros((self.frame_h, self.frame_w), dtype=np.uint32)
        metrics = self.abi.FireCudaFrameMetrics()
        self._check(self.lib.oracle_step(self.h, bgra.ctypes.data, ctypes.byref(settings), ctypes.byref(metrics), mode),
                    "oracle_step")
        return bgra, metrics

    def last_metrics(self):
        sums = (ctypes.c_double * 21)()
        words = (ctypes.c_int * 10)()
        self.lib.oracle_last_metrics(self.h, sums, words)
        return np.array(list(sums), dtype=np.float64), np.array(list(words), dtype=np.int32)

    def times(self):
        t, r, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        self.lib.oracle_times(self.h, ctypes.byref(t), ctypes.byref(r), ctypes.byref(f))
        return t.value, r.value, f.value

    def set_times(self, sim_time: float, render_time: float, frame_index: int) -> None:
        self.lib.oracle_set_times(self.h, sim_time, render_time, frame_index)

    @staticmethod
    def set_threads(n: int) -> None:
        if _LIB is not None:
            _LIB.oracle_set_threads(n)


_CFG_READY = False


def _cfg_lib(abi):
    global _CFG_READY
    L = lib(abi)
    if not _CFG_READY:
        P = ctypes.POINTER(abi.FirePhysicsParams)
        L.cfg_oracle_create.restype = ctypes.c_void_p
        L.cfg_oracle_create.argtypes = [ctypes.c_int] * 6
        L.cfg_oracle_destroy.argtypes = [ctypes.c_void_p]
        L.cfg_oracle_set_physics.argtypes = [ctypes.c_void_p, P]
        L.cfg_oracle_set_pressure_solver.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]
        L.cfg_oracle_set_multigrid.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        L.cfg_oracle_multigrid_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]
        L.cfg_oracle_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.cfg_oracle_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.cfg_oracle_get_field_f64.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        L.cfg_oracle_stages.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.cfg_oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.cfg_oracle_step_count.restype = ctypes.c_ulonglong
        L.cfg_oracle_step_count.argtypes = [ctypes.c_void_p]
        L.cfg_oracle_last_error.restype = ctypes.c_char_p
        _CFG_READY = True
    return L


class ConfigOracle:
    """The config physics (FirePhysicsParams.mode 1) on the CPU, from an empty
    scene. precision 'f32' (the product's rounding) or 'f64'."""

    FIELDS = ("heat", "fuel", "soot", "pressure", "divergence", "u", "v", "w", "hdr", "config_transmittance")

    def __init__(self, abi, frame_w: int, frame_h: int, nx: int, ny: int, nz: int, precision: str = "f32"):
        self.abi = abi
        self.lib = _cfg_lib(abi)
        self.h = self.lib.cfg_oracle_create(0 if precision == "f32" else 1, frame_w, frame_h, nx, ny, nz)
        if not self.h:
            raise RuntimeError(self.lib.cfg_oracle_last_error().decode())
        self.frame_w, self.frame_h = frame_w, frame_h
        self.nx, self.ny, self.nz = nx, ny, nz

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.cfg_oracle_destroy(h)
            self.h = None

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed: {self.lib.cfg_oracle_last_error().decode()}")

    def shape_of(self, name: str):
        nx, ny, nz = self.nx, self.ny, self.nz
        return {
            "u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx),
            "hdr": (self.frame_h, self.frame_w, 4),
            "config_transmittance": ((nz + 1) // 2, (ny + 1) // 2, (nx + 1) // 2),
        }.get(name, (nz, ny, nx))

    def set_physics(self, params) -> None:
        self._check(self.lib.cfg_oracle_set_physics(self.h, ctypes.byref(params)), "set_physics")

    def set_pressure_solver(self, iterations: int, omega: float) -> None:
        self.lib.cfg_oracle_set_pressure_solver(self.h, iterations, omega)

    def set_multigrid(self, max_cycles: int, pre_smooth: int = 2, post_smooth: int = 2, tolerance: float = 0.0) -> None:
        self.lib.cfg_oracle_set_multigrid(self.h, max_cycles, pre_smooth, post_smooth, tolerance)

    def multigrid_stats(self):
        c, m = ctypes.c_int(), ctypes.c_float()
        self.lib.cfg_oracle_multigrid_stats(self.h, ctypes.byref(c), ctypes.byref(m))
        return c.value, m.value

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape_of(name), dtype=np.float32)
        self._check(self.lib.cfg_oracle_get_field(self.h, self.abi.FIELDS[name], out.ctypes.data, out.nbytes), f"get {name}")
        return out

    def get64(self, name: str) -> np.ndarray:
        out = np.empty(self.shape_of(name), dtype=np.float64)
        self._check(self.lib.cfg_oracle_get_field_f64(self.h, self.abi.FIELDS[name], out.ctypes.data, out.size), f"get64 {name}")
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(self.shape_of(name))
        self._check(self.lib.cfg_oracle_set_field(self.h, self.abi.FIELDS[name], a.ctypes.data, a.nbytes), f"set {name}")

    def stages(self, first: str, last: str) -> None:
        s = self.abi.STAGES
        self._check(self.lib.cfg_oracle_stages(self.h, s[first], s[last]), f"stages {first}..{last}")

    def step(self, render: bool = False) -> None:
        self._check(self.lib.cfg_oracle_step(self.h, 1 if render else 0), "step")

    def step_count(self) -> int:
        return int(self.lib.cfg_oracle_step_count(self.h))
