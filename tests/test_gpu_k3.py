"""The reference's interior views (K3) through the CUDA path: the three fixture files the reference
writes (tests/golden/k3-{plan,panorama,fisheye}.rsb) render at 4 spp to the film hashes it pins
(engine/crates/rt-core/src/render/k3_tests.rs:17-22): an orthographic plan with its ceiling hidden
to the camera, an equirectangular panorama and an equidistant fisheye whose corners see nothing,
all lit through a thin pane by the physical sky. The exact passes of the fisheye give the
background where it sees nothing and the distance (not the depth along an axis) elsewhere."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


@pytest.mark.parametrize("view", ["plan", "panorama", "fisheye"])
def test_k3_views_have_the_pinned_hashes(rtg, pins, view):
    s = rtg.Scene((GOLDEN / f"k3-{view}.rsb").read_bytes())
    f = s.film()
    f.render(0, 1)
    f.render(1, 3)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"][f"k3_{view}_4spp"]
    g = s.film()
    g.render_noalloc(0, 4)
    assert rtg.fnv1a(g.resolve()) == pins["film_hashes"][f"k3_{view}_4spp"]


def test_fisheye_paths_and_passes_match_the_oracle(rtg, oracle_lib):
    data = (GOLDEN / "k3-fisheye.rsb").read_bytes()
    g, o = rtg.Scene(data), oracle_lib.OracleScene(data)
    xys = np.stack(np.meshgrid(np.arange(g.width), np.arange(g.height), indexing="xy"), -1).reshape(-1, 2)
    xys = np.concatenate([xys, np.full((len(xys), 1), 5)], 1).astype(np.uint32)
    got, want = g.render_paths(xys), o.paths(xys)
    assert np.allclose(got[:, :4], want[:, :4], rtol=1.0e-4, atol=1.0e-6)
    dark = np.all(got[:, :3] == 0.0, axis=1)
    assert dark[0] and dark[g.width - 1]  # the corners, beyond 180 degrees, bring no light
    st, words = rtg.tile_passes(g.handle, 0, 0, g.width, g.height, 0x1E)  # normal, depth, part, material
    assert st == rtg.STATUS_OK
    n = g.width * g.height
    normal, depth, part, material = o.passes()
    assert np.array_equal(words[:3 * n], np.ascontiguousarray(normal, np.float32).view(np.uint32).reshape(-1))
    assert np.array_equal(words[3 * n:4 * n], np.ascontiguousarray(depth, np.float32).view(np.uint32).reshape(-1))
    assert np.array_equal(words[4 * n:5 * n], part.reshape(-1)) and np.array_equal(words[5 * n:6 * n], material.reshape(-1))
    assert np.isinf(depth[0, 0]) and part[0, 0] == 0  # a corner: the background
