"""Shared test setup: markers, the package loader and the oracle/reference bindings."""
from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "native-firesim_b200"
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU test")


def load_package():
    """Import native-firesim_b200/ (a directory name with a hyphen) as `firesim_b200`."""
    if "firesim_b200" in sys.modules:
        return sys.modules["firesim_b200"]
    spec = importlib.util.spec_from_file_location("firesim_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["firesim_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def abi(pkg):
    return pkg.abi


def load_golden(name: str):
    data = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(bytes(data["__meta__"]).decode())
    return data, meta


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as om  # noqa: PLC0415
    return om


STATE_FIELDS = ["heat", "fuel", "oxygen", "soot", "char", "ash", "pyrolysis", "progress", "turbulence_energy",
                "soot_optics", "pressure", "divergence", "u", "v", "w", "scene_light", "scene_shadow"]
STAGE_OUTPUTS = {
    "advect_velocity": ["u", "v", "w"],
    "advect_react": STATE_FIELDS[:10],
    "force": ["u", "v", "w"],
    "velocity_boundary": ["u", "v", "w"],
    "divergence": ["divergence", "pressure"],
    "pressure_sor": ["pressure"],
    "subtract": ["u", "v", "w"],
    "wall_boundary": ["u", "v", "w"],
    "light_build": ["scene_light", "scene_shadow"],
    "light_propagate": ["scene_light"],
    "render": ["hdr"],
    "embers": ["hdr"],
    "tonemap": ["bgra"],
    "overlay": ["bgra"],
    "metrics": ["divergence_after"],
}
RENDER_STAGES = ("render", "embers", "tonemap", "overlay")
