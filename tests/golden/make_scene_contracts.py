"""Copies the reference's scene contracts (scene.json, emitter-mask.json of the
three scenes, about 1 KB each) into tests/golden/scene_contracts/ so the
contract tests run without the reference checkout.

Usage: python tests/golden/make_scene_contracts.py <native-firesim checkout>
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "scene_contracts"


def main() -> int:
    if len(sys.argv) != 2:
        print(__doc__.strip().splitlines()[-1], file=sys.stderr)
        return 2
    ref = Path(sys.argv[1]) / "assets" / "fire-scenes"
    for asset in ("room", "campfire", "gas-burner-aver1"):
        (OUT / asset).mkdir(parents=True, exist_ok=True)
        for name in ("scene.json", "emitter-mask.json"):
            src = ref / asset / name
            if src.exists():
                shutil.copyfile(src, OUT / asset / name)
                print("copied", src)
    return 0


if __name__ == "__main__":
    sys.exit(main())
