"""The reference's interior views (K3) on the oracle: the three fixture files the reference writes
(`rt --write-k3-{plan,panorama,fisheye}-example`, kept in tests/golden/) render at 4 spp to the
film hashes the reference pins (engine/crates/rt-core/src/render/k3_tests.rs:17-22). Together they
pin the orthographic plan with its ceiling hidden to the camera, the equirectangular panorama, the
equidistant fisheye (whose corners, beyond 180 degrees, see nothing), the physical sky seen
through a thin pane and the exterior factor."""
from pathlib import Path

import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("view", ["plan", "panorama", "fisheye"])
def test_k3_views_have_the_pinned_hashes(oracle_lib, pins, view):
    s = oracle_lib.OracleScene((GOLDEN / f"k3-{view}.rsb").read_bytes())
    rgb, w, _, _, _ = s.render_film(0, 4, tile=32, threads=8)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"][f"k3_{view}_4spp"]
