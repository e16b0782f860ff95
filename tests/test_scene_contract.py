"""fireCudaApplySceneContract against the reference worker's contract rules (CPU).

The reference's worker fills FireSettings' emitter fields from
assets/fire-scenes/<id>/scene.json and emitter-mask.json with a first-
occurrence key scanner (src/main.cpp:1148-1264, :1397-1476, :433-447).  This
test restates those rules independently in Python (regular expressions over
the raw text, float32 arithmetic) and compares every field bit for bit, on the
reference's three contracts (copied by tests/golden/make_scene_contracts.py)
and on synthetic contracts that exercise each rule.  Host-only: no GPU.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

CONTRACTS = Path(__file__).resolve().parent / "golden" / "scene_contracts"
ASSETS = {0: "room", 1: "campfire", 2: "gas-burner-aver1"}
f32 = np.float32


def _after_key(text: str, key: str) -> int:
    m = text.find(f'"{key}"')
    return m


def _number(text: str, key: str):
    at = _after_key(text, key)
    if at < 0:
        return None
    colon = text.find(":", at + len(key) + 2)
    if colon < 0:
        return None
    m = re.match(r"\s*([-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?)", text[colon + 1:])
    return f32(float(m.group(1))) if m else None


def _span(text: str, key: str, open_c: str, close_c: str, strings: bool) -> str:
    at = _after_key(text, key)
    if at < 0:
        return ""
    start = text.find(open_c, at)
    if start < 0:
        return ""
    depth, in_str, esc = 0, False, False
    for i in range(start, len(text)):
        c = text[i]
        if strings:
            if esc:
                esc = False
                continue
            if c == "\\":
                esc = in_str
                continue
            if c == '"':
                in_str = not in_str
                continue
            if in_str:
                continue
        if c == open_c:
            depth += 1
        elif c == close_c:
            depth -= 1
            if depth == 0:
                return text[start:i + 1]
    return ""


def _numbers(span: str):
    return [f32(float(m)) for m in re.findall(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?", span)]


def _triplet(text, key, fallback):
    v = _numbers(_span(text, key, "[", "]", False))
    return v[:3] if len(v) >= 3 else [f32(x) for x in fallback]


def expected(scene: int, root):
    e = dict(cx=f32(0), cz=f32(0), hn=f32(0), hb=f32(0.06), r=f32(0.48), n=0, bx=[f32(0)] * 4, by=[f32(0)] * 4, bz=[f32(0)] * 4)
    d = None if root is None else Path(root) / ASSETS[scene]
    text = (d / "scene.json").read_text() if d is not None and (d / "scene.json").exists() else ""
    if text:
        src = _span(text, "emitter", "{", "}", True) or text
        c = _triplet(src, "centerMeters", (0.0, 0.02, 0.0))
        e["cx"], e["cz"], e["hn"] = c[0], c[2], f32((c[1] - f32(0.02)) / f32(2.03))
        v = _number(src, "radiusMeters")
        if v is not None:
            e["r"] = v
        v = _number(src, "heightBandMeters")
        if v is not None:
            e["hb"] = f32(v / f32(2.03))
    elif scene == 1:
        e.update(r=f32(0.32), hn=f32((f32(0.045) - f32(0.02)) / f32(2.03)), hb=f32(f32(0.20) / f32(2.03)))
    elif scene == 2:
        e.update(r=f32(0.24), hn=f32((f32(0.138) - f32(0.02)) / f32(2.03)), hb=f32(f32(0.105) / f32(2.03)))
    if scene == 0 or d is None or not (d / "emitter-mask.json").exists():
        return e
    mask = (d / "emitter-mask.json").read_text()
    shift = _triplet(text, "translationMeters", (0.0, -0.24 if scene == 2 else 0.0, 0.0))
    for key, field in (("centerXMeters", "cx"), ("centerZMeters", "cz")):
        v = _number(mask, key)
        if v is not None:
            e[field] = v
    v = _number(mask, "centerYMeters")
    if v is None:
        v = _number(mask, "worldHeightMeters")
    if v is not None:
        e["hn"] = f32((v - f32(0.02)) / f32(2.03))
    v = _number(mask, "heightBandMeters")
    if v is not None:
        e["hb"] = f32(v / f32(2.03))
    v = _number(mask, "radiusMeters")
    if v is not None:
        e["r"] = v
    else:
        frac, w, dep = _number(mask, "radiusFraction"), _number(mask, "width"), _number(mask, "depth")
        if frac is not None and w is not None and dep is not None:
            e["r"] = f32(frac * max(w, dep))
    b = _numbers(_span(mask, "burnerCentersMeters", "[", "]", False))
    e["n"] = min(4, len(b) // 3)
    e["bx"], e["by"], e["bz"] = list(e["bx"]), list(e["by"]), list(e["bz"])
    for i in range(e["n"]):
        e["bx"][i] = f32(b[3 * i] + shift[0])
        e["by"][i] = f32(b[3 * i + 1] + shift[1])
        e["bz"][i] = f32(b[3 * i + 2] + shift[2])
    if scene == 2 and e["n"] > 0:
        e["hn"] = f32((e["by"][0] - f32(0.02)) / f32(2.03))
    return e


def _applied(pkg, scene, root):
    s = pkg.abi.FireSettings()
    pkg.firesim.apply_scene_contract(scene, root, s)
    return dict(cx=f32(s.emitterCenterX), cz=f32(s.emitterCenterZ), hn=f32(s.emitterHeightNorm), hb=f32(s.emitterHeightBandNorm),
                r=f32(s.emitterRadius), n=s.burnerCenterCount, bx=[f32(x) for x in s.burnerCenterX],
                by=[f32(x) for x in s.burnerCenterY], bz=[f32(x) for x in s.burnerCenterZ])


def _same(a, b):
    for k in a:
        x, y = np.asarray(a[k], dtype=np.float32), np.asarray(b[k], dtype=np.float32)
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (k, a[k], b[k])


@pytest.mark.parametrize("scene", [0, 1, 2])
@pytest.mark.parametrize("with_files", [True, False])
def test_contract_matches_reference_rules(scene, with_files, pkg):
    root = CONTRACTS if with_files else None
    _same(_applied(pkg, scene, root), expected(scene, root))


def test_gas_burner_known_values(pkg):
    """Hand-read values of the gas burner: radius and centre from
    "derivedEmitter", height band from "emitterHint" (its first occurrence),
    height from the selected burner's centre shifted by the mesh translation."""
    got = _applied(pkg, 2, CONTRACTS)
    assert got["n"] == 1
    assert got["r"] == f32(0.13822224736213684)
    assert got["cx"] == f32(0.1980201154947281) and got["cz"] == f32(0.23754769563674927)
    assert got["hb"] == f32(f32(0.105) / f32(2.03))
    assert got["by"][0] == f32(f32(0.37620601058006287) + f32(-0.24))
    assert got["hn"] == f32((got["by"][0] - f32(0.02)) / f32(2.03))


def test_synthetic_contract_rules(pkg, tmp_path):
    """First occurrence wins even inside nested objects; radiusFraction x max(width, depth);
    worldHeightMeters when centerYMeters is absent; at most four burners."""
    d = tmp_path / "campfire"
    d.mkdir()
    (d / "scene.json").write_text('{"meshTransform": {"translationMeters": [0.5, 0.25, -0.5]},'
                                  ' "emitter": {"centerMeters": [0.1, 0.3, -0.2], "heightBandMeters": 0.4}}')
    (d / "emitter-mask.json").write_text('{"hint": {"heightBandMeters": 0.05, "radiusFraction": 0.5},'
                                         ' "size": {"width": 0.6, "depth": 0.8}, "worldHeightMeters": 0.3,'
                                         ' "burnerCentersMeters": [[1,2,3],[4,5,6],[7,8,9],[1,1,1],[2,2,2]],'
                                         ' "later": {"heightBandMeters": 9.0}}')
    got = _applied(pkg, 1, tmp_path)
    _same(got, expected(1, tmp_path))
    assert got["n"] == 4 and got["r"] == f32(f32(0.5) * f32(0.8))
    assert got["hb"] == f32(f32(0.05) / f32(2.03))
    assert got["bx"][0] == f32(f32(1) + f32(0.5))


def test_null_settings_rejected(pkg):
    lib = pkg.load_library()
    assert not lib.fireCudaApplySceneContract(0, None, None)
    assert "settings pointer was null" in pkg.firesim.last_error()
