"""The resident SOR's brick-shape autotuner (needs a GPU): where both brick
shapes fit co-resident, the first solve of a grid times one solve with each
and keeps the faster.  The result must equal the untuned solve bit for bit,
and the recorded choice must be the faster of the two timings."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(pkg, abi, dims, autotune):
    pkg.set_autotune(autotune)
    sim = pkg.FireSim(64, 32, *dims)
    sim.set_pressure_solver(40, 1.8)
    rng = np.random.default_rng(3)
    d = rng.standard_normal(dims[::-1]).astype(np.float32)
    p0 = (0.1 * rng.standard_normal(dims[::-1])).astype(np.float32)
    sim.set("divergence", d)
    sim.set("pressure", p0)
    sim.stages("pressure_sor", "pressure_sor", abi.FireSettings(), 0.0)
    out = sim.get("pressure"), sim.pressure_path_used()
    sim.close()
    return out


@pytest.mark.parametrize("dims", [(96, 96, 96), (64, 80, 48)])
def test_autotuned_resident_solve_equals_the_fixed_rule(pkg, abi, dims):
    fixed, path_fixed = _solve(pkg, abi, dims, False)
    tuned, path_tuned = _solve(pkg, abi, dims, True)
    pkg.set_autotune(True)
    assert path_fixed == 2 and path_tuned == 2
    np.testing.assert_array_equal(tuned.view(np.uint32), fixed.view(np.uint32))
    rec = pkg.tuned_brick(*dims)
    assert rec is not None, "both brick shapes fit here, so the first solve should have been timed"
    bx, ms32, ms16 = rec
    assert bx in (16, 32) and ms32 > 0 and ms16 > 0
    assert (bx == 32) == (ms32 <= ms16)
    print(f"{dims}: 32x16x16 {ms32:.3f} ms, 16x16x16 {ms16:.3f} ms -> {bx}")
