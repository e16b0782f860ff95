"""The C ABI of libfiresim_b200.so without a GPU: symbols, struct layouts, error paths.

No test here launches device work; the calls exercised return before any CUDA
call, exactly as the reference's entry points do when uninitialised.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from conftest import ROOT

HEADERS = [ROOT / "include" / "fire_cuda.h", ROOT / "include" / "fire_ext.h"]


def declared_symbols() -> set[str]:
    names = set()
    for h in HEADERS:
        names |= set(re.findall(r"^FIRE_API [^(]*?\b(fire\w+)\(", h.read_text(), flags=re.M))
    return names


def test_headers_declare_the_reference_abi():
    names = declared_symbols()
    reference = {
        "fireCudaInitialize", "fireCudaStepAndRender", "fireCudaStepAndRenderMeasured", "fireCudaSelectDeviceForD3D11",
        "fireCudaRegisterD3D11Texture", "fireCudaRegisterD3D11TextureSlot", "fireCudaSetD3D11TextureSlot",
        "fireCudaStepD3D11", "fireCudaStepAndRenderD3D11", "fireCudaStepAndRenderD3D11Measured", "fireCudaRenderD3D11",
        "fireCudaUnregisterD3D11Texture", "fireCudaSynchronize", "fireCudaReset", "fireCudaGetDiagnostics",
        "fireCudaShutdown", "fireCudaLastError",
    }
    assert reference <= names, reference - names


@pytest.mark.parametrize("precision", ["f32", "f16", "bf16", "checked"])
def test_library_exports_every_declared_symbol(pkg, precision):
    """Every build (FP32, FP16 and BF16 storage, bounds-checking) exports the whole declared ABI."""
    lib = pkg.load_library(precision)
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), name


def test_struct_layouts(abi):
    # Byte sizes of the reference structs (src/fire_cuda.h:5-100) on LP64.
    assert ctypes.sizeof(abi.FireCudaDiagnostics) == 6 * 4 + 8 + 128
    assert ctypes.sizeof(abi.FireCudaFrameMetrics) == 6 * 4 + 40 * 4
    assert ctypes.sizeof(abi.FireSettings) == 32 * 4 + 3 * 16
    assert abi.FireSettings().showGizmos == 1 and abi.FireSettings().raymarchSteps == 56


def test_uninitialised_calls_fail_with_reference_messages(pkg, abi):
    lib = pkg.load_library()
    lib.fireCudaShutdown()
    s = abi.FireSettings()
    buf = (ctypes.c_uint32 * 4)()
    assert not lib.fireCudaStepAndRender(buf, ctypes.byref(s))
    assert pkg.firesim.last_error() == "CUDA renderer is not initialized."
    assert not lib.fireCudaStepAndRenderMeasured(buf, ctypes.byref(s), None)
    assert pkg.firesim.last_error() == "Metrics output pointer was null."
    assert not lib.fireCudaReset()
    assert not lib.fireCudaRunStages(0, 0, ctypes.byref(s), 0.0)
    assert not lib.fireCudaGetDiagnostics(None)
    assert pkg.firesim.last_error() == "Diagnostics output pointer was null."


def test_guard_checks_report_the_default_build(pkg):
    """Outside the FIRE_BOUNDS_CHECK build the guard entry points say so and
    make no CUDA call."""
    lib = pkg.load_library()
    n = ctypes.c_int(7)
    assert not lib.fireCudaCheckGuards(ctypes.byref(n))
    assert n.value == -1
    assert "FIRE_BOUNDS_CHECK" in pkg.firesim.last_error()
    assert pkg.check_guards("f32") == -1
    assert not lib.fireCudaPlantGuardByte(b"pressure", 0)
    assert "FIRE_BOUNDS_CHECK" in pkg.firesim.last_error()


def test_d3d11_entry_points_report_headless(pkg):
    lib = pkg.load_library()
    assert not lib.fireCudaSelectDeviceForD3D11(ctypes.c_void_p(1))
    assert "D3D11 unavailable on headless build" in pkg.firesim.last_error()
    assert not lib.fireCudaRegisterD3D11Texture(ctypes.c_void_p(1))
    assert not lib.fireCudaRegisterD3D11TextureSlot(0, ctypes.c_void_p(1))
    assert "fireCudaRegisterHdrBufferSlot" in pkg.firesim.last_error()


def test_library_has_no_oracle_dependency():
    """The product neither links nor names the oracle."""
    import subprocess
    for name in ("libfiresim_b200.so", "libfiresim_b200_f16.so", "libfiresim_b200_bf16.so", "libfiresim_b200_checked.so"):
        lib = ROOT / "native-firesim_b200" / name
        needed = subprocess.run(["readelf", "-d", str(lib)], capture_output=True, text=True).stdout
        assert "oracle" not in needed and "fire_ref" not in needed
    for src in (ROOT / "native-firesim_b200").rglob("*"):
        if src.suffix in (".cu", ".cuh", ".h", ".py", ".cpp"):
            assert "oracle" not in src.read_text().lower(), src


@pytest.mark.parametrize("struct", ["FireSettings", "FireCudaFrameMetrics", "FireEmitterDisk", "FirePhysicsParams",
                                    "FireServeRequest", "FireServeReport"])
def test_struct_offsets_match_the_header(abi, struct, tmp_path):
    """Every field of the ctypes mirror sits at the offset g++ gives it from include/*.h."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not found")
    cls = getattr(abi, struct)
    lines = [f'std::printf("size %zu\\n", sizeof({struct}));']
    for name, _ in cls._fields_:
        lines.append(f'std::printf("{name} %zu\\n", offsetof({struct}, {name}));')
    src = tmp_path / "probe.cpp"
    src.write_text('#include <cstddef>\n#include <cstdio>\n#include "fire_ext.h"\nint main() {\n' + "\n".join(lines) +
                   "\nreturn 0;\n}\n")
    exe = tmp_path / "probe"
    subprocess.run([cxx, "-std=c++17", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    assert int(got["size"]) == ctypes.sizeof(cls)
    for name, _ in cls._fields_:
        assert int(got[name]) == getattr(cls, name).offset, name


def test_callers_of_the_reference_header_link_unchanged(tmp_path):
    """A C++ caller compiled against declarations with the reference header's
    C++ linkage (src/fire_cuda.h:102-118) links against libfiresim_b200.so
    through the exported mangled aliases and gets the reference's messages."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not found")
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include <cstdint>
#include <cstdio>
#include <cstring>
struct FireSettings { unsigned char bytes[176]; };
struct FireCudaFrameMetrics; struct FireCudaDiagnostics;
bool fireCudaInitialize(int, int, int, int);
bool fireCudaStepAndRender(std::uint32_t*, const FireSettings&);
bool fireCudaStepAndRenderMeasured(std::uint32_t*, const FireSettings&, FireCudaFrameMetrics*);
bool fireCudaSelectDeviceForD3D11(void*);
bool fireCudaRegisterD3D11Texture(void*);
bool fireCudaRegisterD3D11TextureSlot(int, void*);
bool fireCudaSetD3D11TextureSlot(int);
bool fireCudaStepD3D11(const FireSettings&);
bool fireCudaStepAndRenderD3D11(const FireSettings&);
bool fireCudaStepAndRenderD3D11Measured(const FireSettings&, FireCudaFrameMetrics*);
bool fireCudaRenderD3D11(const FireSettings&);
void fireCudaUnregisterD3D11Texture();
bool fireCudaSynchronize();
bool fireCudaReset();
bool fireCudaGetDiagnostics(FireCudaDiagnostics*);
void fireCudaShutdown();
const char* fireCudaLastError();
int main() {
    void* all[] = {(void*)&fireCudaInitialize, (void*)&fireCudaStepAndRenderMeasured, (void*)&fireCudaRegisterD3D11TextureSlot,
                   (void*)&fireCudaSetD3D11TextureSlot, (void*)&fireCudaStepD3D11, (void*)&fireCudaStepAndRenderD3D11,
                   (void*)&fireCudaStepAndRenderD3D11Measured, (void*)&fireCudaRenderD3D11, (void*)&fireCudaUnregisterD3D11Texture,
                   (void*)&fireCudaSynchronize, (void*)&fireCudaGetDiagnostics};
    for (void* f : all) if (f == nullptr) return 2;
    fireCudaShutdown();
    FireSettings s{};
    std::uint32_t px[4] = {};
    if (fireCudaStepAndRender(px, s)) return 3;
    std::printf("%s\n", fireCudaLastError());
    if (fireCudaReset()) return 4;
    if (fireCudaSelectDeviceForD3D11(nullptr)) return 5;
    std::printf("%s\n", fireCudaLastError());
    if (fireCudaRegisterD3D11Texture(nullptr)) return 6;
    return 0;
}
''')
    lib_dir = ROOT / "native-firesim_b200"
    exe = tmp_path / "caller"
    subprocess.run([cxx, "-std=c++17", str(src), "-o", str(exe), f"-L{lib_dir}", "-lfiresim_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    lines = out.stdout.splitlines()
    assert lines[0] == "CUDA renderer is not initialized."
    assert "D3D11 unavailable on headless build" in lines[1]
