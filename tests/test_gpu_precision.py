"""Half storage of the transported fields (libfiresim_b200_f16.so and
libfiresim_b200_bf16.so; needs a GPU).

These builds store the ten scalars and the three face grids as IEEE half or
bfloat16 (FP32 arithmetic; pressure, divergence, forcing, light and frames
FP32).  Their error is stated two ways:
  * against the FP32 build on identical inputs (the same noise, so the
    difference is the storage alone): relative L2 per field after 20 steps;
  * against the FP64 CPU oracle, beside the FP32 build's own error there.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["heat", "fuel", "oxygen", "soot", "progress", "u", "v", "w", "pressure"]


def _run(pkg, abi, precision, n, steps, metrics=False):
    sim = pkg.FireSim(64, 48, n, n, n, precision=precision)
    m = None
    for f in range(steps):
        s = abi.validation_settings(f, width=64, height=48)
        s.reset = 1 if f == 0 else 0
        if metrics:
            _, m = sim.step_and_render(s, metrics=True)
        else:
            sim.step(s)
    sim.synchronize()
    out = {k: sim.get(k).astype(np.float64) for k in FIELDS}
    sim.close()
    return out, (m.as_dict() if m is not None else None)


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# precision -> (field rel L2 bound, frame-sum rel bound); measured at 64^3 after
# 20 steps: f16 4e-5 .. 1.5e-3 and sums within 0.02%; bf16 4e-4 .. 1.2e-2 and
# sums within 0.3%.
BOUNDS = {"f16": (5e-3, 1e-3), "bf16": (3e-2, 1e-2)}


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_half_storage_vs_f32(pkg, abi, precision):
    """64^3, 20 validation steps with a render each, against the FP32 build:
    every field and the frame sums within the bounds above, the post-projection
    divergence L2 within 1%."""
    field_bound, sum_bound = BOUNDS[precision]
    a, ma = _run(pkg, abi, "f32", 64, 20, metrics=True)
    b, mb = _run(pkg, abi, precision, 64, 20, metrics=True)
    for k in FIELDS:
        assert _rel_l2(b[k], a[k]) <= field_bound, (k, _rel_l2(b[k], a[k]))
    for k in ("heatSum", "fuelSum", "sootSum"):
        assert mb[k] == pytest.approx(ma[k], rel=sum_bound), k
    assert mb["divergenceAfterL2"] == pytest.approx(ma["divergenceAfterL2"], rel=1e-2)


def test_half_and_f32_vs_fp64_oracle(pkg, abi, oracle_mod):
    """48^3, 12 steps against the FP64 oracle: the FP16 build's error is at most
    1.25x the FP32 build's own plus 1e-3 (measured: 3-10% above it), the BF16
    build's at most 3x plus 3e-3 (measured: 2-2.5x)."""
    n, steps = 48, 12
    o = oracle_mod.OracleFire(abi, 64, 48, n, n, n, precision="f64")
    for f in range(steps):
        s = abi.validation_settings(f, width=64, height=48)
        s.reset = 1 if f == 0 else 0
        o.step(s, mode=2)
    ref = {k: o.get64(k) for k in FIELDS}
    e32 = {k: _rel_l2(v, ref[k]) for k, v in _run(pkg, abi, "f32", n, steps)[0].items()}
    e16 = {k: _rel_l2(v, ref[k]) for k, v in _run(pkg, abi, "f16", n, steps)[0].items()}
    ebf = {k: _rel_l2(v, ref[k]) for k, v in _run(pkg, abi, "bf16", n, steps)[0].items()}
    for k in FIELDS:
        assert e16[k] <= 1.25 * e32[k] + 1e-3, (k, e16[k], e32[k])
        assert ebf[k] <= 3.0 * e32[k] + 3e-3, (k, ebf[k], e32[k])


def test_f16_scenes_alone_equal_batched(pkg, abi):
    """The FP16 build keeps the determinism of the FP32 one: a scene stepped
    alone equals the same scene stepped beside two others, bit for bit."""
    sizes = [(24, 28, 20), (32, 32, 32), (40, 24, 36)]
    scenes = [pkg.Scene(64, 48, *d, precision="f16") for d in sizes]
    for f in range(6):
        sets = []
        for i in range(3):
            s = abi.validation_settings(f, scene=i, width=64, height=48)
            s.reset = 1 if f == 0 else 0
            sets.append(s)
        pkg.batch_step(scenes, sets)
    alone = pkg.Scene(64, 48, *sizes[1], precision="f16")
    for f in range(6):
        s = abi.validation_settings(f, scene=1, width=64, height=48)
        s.reset = 1 if f == 0 else 0
        alone.step(s)
    for k in ("heat", "u", "pressure"):
        np.testing.assert_array_equal(scenes[1].get(k).view(np.uint32), alone.get(k).view(np.uint32), err_msg=k)
    for sc in scenes + [alone]:
        sc.close()
