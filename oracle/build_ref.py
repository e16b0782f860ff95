"""Build recipe for oracle/_ref/libfire_ref.so -- test infrastructure only.

Compiles native-firesim's own CUDA translation unit, src/fire_cuda.cu, from
where it lies under the reference checkout, together with oracle/ref_harness.cu.
The reference TU needs <d3d11.h> and <cuda_d3d11_interop.h>, which do not exist
on Linux.  Instead of standing in for them, this recipe writes a derived copy
into oracle/_ref/ with exactly these pieces removed:

  * the two #include lines of the D3D11 headers (src/fire_cuda.cu:4, :7);
  * the three D3D11-only entry points fireCudaSelectDeviceForD3D11,
    fireCudaRegisterD3D11Texture and fireCudaRegisterD3D11TextureSlot
    (src/fire_cuda.cu:3563-3601).

Everything else -- every kernel, helper and the host sequencing -- is compiled
as written.  Outputs go only to oracle/_ref/ (git-ignored).  The reference is
never modified and none of its sources are committed.

Usage: python oracle/build_ref.py --reference /path/to/native-firesim
       (or FIRESIM_REFERENCE=/path/to/native-firesim python oracle/build_ref.py)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"

def reference_root(explicit: str | None = None) -> Path | None:
    """The native-firesim checkout: the explicit path, else $FIRESIM_REFERENCE, else None."""
    value = explicit or os.environ.get("FIRESIM_REFERENCE")
    return Path(value) if value else None


def derive_headless_source(reference: Path) -> str:
    src = (reference / "src" / "fire_cuda.cu").read_text().split("\n")
    out = []
    skipping = False
    removed_includes = 0
    removed_lines = 0
    for line in src:
        if line.startswith("#include <d3d11.h>") or line.startswith("#include <cuda_d3d11_interop.h>"):
            removed_includes += 1
            continue
        if line.startswith("bool fireCudaSelectDeviceForD3D11("):
            skipping = True
        if line.startswith("bool fireCudaSetD3D11TextureSlot("):
            skipping = False
        if skipping:
            removed_lines += 1
            continue
        out.append(line)
    if removed_includes != 2 or not (30 <= removed_lines <= 50):
        raise RuntimeError(
            f"unexpected reference layout: removed {removed_includes} includes, {removed_lines} lines")
    return "\n".join(out)


def build(reference: Path, verbose: bool = False) -> Path:
    if not (reference / "src" / "fire_cuda.cu").exists():
        raise FileNotFoundError(f"reference sources not found under {reference}")
    OUT.mkdir(parents=True, exist_ok=True)
    derived = OUT / "fire_cuda_headless.cu"
    text = derive_headless_source(reference)
    if not derived.exists() or derived.read_text() != text:
        derived.write_text(text)
    harness = OUT / "ref_harness.cu"
    harness_text = (HERE / "ref_harness.cu").read_text()
    if not harness.exists() or harness.read_text() != harness_text:
        harness.write_text(harness_text)
    lib = OUT / "libfire_ref.so"
    deps = [derived, harness]
    if lib.exists() and all(lib.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return lib
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [
        nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
        "-Xcompiler", "-fPIC", "-shared", "-I", str(reference / "src"), "-I", str(OUT),
        str(harness), "-o", str(lib),
    ]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="native-firesim checkout (default: $FIRESIM_REFERENCE)")
    args = ap.parse_args()
    root = reference_root(args.reference)
    if root is None:
        ap.error("give --reference or set FIRESIM_REFERENCE")
    lib = build(root, verbose=True)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
