"""Build recipe for native-firesim_b200/libfiresim_b200.so (sm_100a).

Compiles every csrc/*.cu (and the host-only csrc/*.cpp) with nvcc for
compute_100a/sm_100a (-O3 -lineinfo),
in parallel, and links them into one shared library next to this file.
nvcc cross-compiles without a GPU, so this runs on a CPU-only host.

Usage: python native-firesim_b200/build.py [--force] [--ptxas-verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OBJ = HERE / "_build"
LIB = HERE / "libfiresim_b200.so"
# The reduced-storage variants: the same sources with -DFIRE_STORAGE_F16 / -DFIRE_STORAGE_BF16.
VARIANTS = {
    "f32": (HERE / "_build", HERE / "libfiresim_b200.so", []),
    "f16": (HERE / "_build_f16", HERE / "libfiresim_b200_f16.so", ["-DFIRE_STORAGE_F16"]),
    "bf16": (HERE / "_build_bf16", HERE / "libfiresim_b200_bf16.so", ["-DFIRE_STORAGE_BF16"]),
    # FP32 storage with guard zones around every device buffer (csrc/fire_guard.h).
    "checked": (HERE / "_build_checked", HERE / "libfiresim_b200_checked.so", ["-DFIRE_BOUNDS_CHECK"]),
}
INCLUDE = HERE.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr"]
# Per-file flags: the config-physics and multigrid kernels round every product
# and sum as written (no FMA contraction), so their CPU restatement can match
# them bit for bit.
FILE_FLAGS = {"fire_config.cu": ["-fmad=false"], "fire_mg.cu": ["-fmad=false"]}


def _nvcc() -> str:
    return os.environ.get("NVCC", "nvcc")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _compile(src: Path, force: bool, verbose_ptxas: bool, variant: str = "f32") -> tuple[Path, str]:
    obj = VARIANTS[variant][0] / (src.stem + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep and not verbose_ptxas:
        return obj, ""
    cmd = [_nvcc(), *ARCH, *CUFLAGS, *FILE_FLAGS.get(src.name, []), *VARIANTS[variant][2], "-I", str(INCLUDE), "-c", str(src), "-o",
           str(obj)]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def _build_variant(variant: str, force: bool, verbose_ptxas: bool, quiet: bool) -> Path:
    objdir, lib, _ = VARIANTS[variant]
    objdir.mkdir(parents=True, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose_ptxas, variant), srcs))
    if verbose_ptxas:
        for _, log in results:
            print(log)
    objs = [o for o, _ in results]
    if force or not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, lib)
        if not quiet:
            print(f"linked {lib}")
    return lib


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True, f16: bool = True) -> Path:
    """Builds the FP32 library (returned) and, unless f16=False, the FP16- and BF16-storage
    variants and the bounds-checking FP32 build."""
    lib = _build_variant("f32", force, verbose_ptxas, quiet)
    if f16:
        _build_variant("f16", force, False, quiet)
        _build_variant("bf16", force, False, quiet)
        _build_variant("checked", force, False, quiet)
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose_ptxas=args.ptxas_verbose, quiet=False))
    return 0


if __name__ == "__main__":
    sys.exit(main())
