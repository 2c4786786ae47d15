"""Shared fixtures. Tests marked ``gpu`` need a B200 and the built native library; the rest run on
CPU (the oracle, the scene builders, the C-ABI exports, the multi-process host logic)."""
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

PINS = json.loads((ROOT / "tests" / "golden" / "reference_pins.json").read_text())


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and repackshot_b200/librtg.so")


@pytest.fixture(scope="session")
def pins():
    return PINS


@pytest.fixture(scope="session")
def example_rsb():
    from repackshot_b200 import scenes
    return scenes.to_rsb(scenes.example_scene())


@pytest.fixture(scope="session")
def cfg0_rsb():
    from repackshot_b200 import scenes
    return scenes.to_rsb(scenes.cfg0_scene())


@pytest.fixture(scope="session")
def small_product_rsb():
    """The product scene's materials, lights and dome on a reduced knot (64 x 32 quads) and a
    small image: every BSDF of the benchmark (conductors, rough glass, Lambert) at oracle speed."""
    from repackshot_b200 import scenes
    return scenes.to_rsb(scenes.product_scene(width=96, height=64, spp=4, depth=12, seg_u=64, seg_v=32))


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    return oracle
