"""ctypes binding for oracle/_ref/libfire_ref.so -- test infrastructure only.

The library is native-firesim's own src/fire_cuda.cu compiled for sm_100a with
oracle/ref_harness.cu (see oracle/build_ref.py).  Only tests and the golden
fixture generator use it; it needs a GPU.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libfire_ref.so"


def available() -> bool:
    return LIB_PATH.exists()


class RefFire:
    """The reference implementation on cuda:0, one global instance per process."""

    def __init__(self, abi, frame_w: int, frame_h: int, nx: int, ny: int, nz: int):
        self.abi = abi
        lib = ctypes.CDLL(str(LIB_PATH))
        self.lib = lib
        lib.ref_init_grid.argtypes = [ctypes.c_int] * 5
        lib.ref_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(abi.FireSettings),
                                 ctypes.POINTER(abi.FireCudaFrameMetrics), ctypes.c_int]
        lib.ref_stages.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(abi.FireSettings), ctypes.c_float]
        lib.ref_field_bytes.restype = ctypes.c_longlong
        lib.ref_get_field.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        lib.ref_set_field.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_last_metrics.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        lib.ref_get_times.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_int)]
        lib.ref_light_dims.argtypes = [ctypes.POINTER(ctypes.c_int)]
        self.frame_w, self.frame_h = frame_w, frame_h
        self.nx, self.ny, self.nz = nx, ny, nz
        self._check(lib.ref_init_grid(frame_w, frame_h, nx, ny, nz), "ref_init_grid")
        dims = (ctypes.c_int * 3)()
        lib.ref_light_dims(dims)
        self.light_dims = tuple(dims)

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.lib.ref_last_error().decode()}")

    def shape_of(self, name: str):
        nx, ny, nz = self.nx, self.ny, self.nz
        lx, ly, lz = self.light_dims
        return {
            "u": (nz, ny, nx + 1), "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx),
            "scene_light": (lz, ly, lx, 4), "scene_shadow": (lz, ly, lx),
            "hdr": (self.frame_h, self.frame_w, 4), "bgra": (self.frame_h, self.frame_w),
        }.get(name, (nz, ny, nx))

    def get(self, name: str) -> np.ndarray:
        fid = self.abi.FIELDS[name]
        dtype = np.uint32 if name == "bgra" else np.float32
        out = np.empty(self.shape_of(name), dtype=dtype)
        self._check(self.lib.ref_get_field(fid, out.ctypes.data, out.nbytes), f"get {name}")
        return out

    def set(self, name: str, arr: np.ndarray) -> None:
        fid = self.abi.FIELDS[name]
        dtype = np.uint32 if name == "bgra" else np.float32
        a = np.ascontiguousarray(arr, dtype=dtype).reshape(self.shape_of(name))
        self._check(self.lib.ref_set_field(fid, a.ctypes.data, a.nbytes), f"set {name}")

    def step(self, settings, mode: int = 1):
        bgra = np.zeros((self.frame_h, self.frame_w), dtype=np.uint32)
        metrics = self.abi.FireCudaFrameMetrics()
        self._check(self.lib.ref_step(bgra.ctypes.data, ctypes.byref(settings), ctypes.byref(metrics), mode),
                    "ref_step")
        return bgra, metrics

    def stages(self, first: str, last: str, settings, time: float) -> None:
        s = self.abi.STAGES
        self._check(self.lib.ref_stages(s[first], s[last], ctypes.byref(settings), time), f"stages {first}..{last}")

    def last_metrics(self):
        sums = (ctypes.c_double * 21)()
        bits = (ctypes.c_int * 10)()
        self.lib.ref_last_metrics(sums, bits)
        return np.array(list(sums), dtype=np.float64), np.array(list(bits), dtype=np.int32)

    def times(self):
        t, r, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        self.lib.ref_get_times(ctypes.byref(t), ctypes.byref(r), ctypes.byref(f))
        return t.value, r.value, f.value

    def close(self):
        self.lib.ref_shutdown()
