"""IES lights on the GPU, through the C ABI: the L5 scene (the example lit by a downlight sphere
and a wall-washer point, the reference's two hand-written profiles) has the reference's pinned
4-sample hash (render.rs:1510-1531); variants (a light outside the sphere that bounds the scene,
whose selection uses its profile towards the scene; profiles turned about their axes; a single IES
light in the dark) have the oracle's film bits, and every tested path is bit-exact.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROFILES = json.loads((Path(__file__).resolve().parent / "golden" / "ies_profiles.json").read_text())


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def l5():
    from repackshot_b200 import scenes
    return scenes.l5_scene(PROFILES["downlight-symmetric"].encode(), PROFILES["wall-washer"].encode())


def test_l5_has_the_pinned_hash(rtg, pins):
    from repackshot_b200 import scenes
    f = rtg.Scene(scenes.to_rsb(l5())).film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["l5_ies_4spp"]


def variant(name):
    s = l5()
    if name == "far washer":
        s.lights[2].position = (-4000.0, -3000.0, 2500.0)
    elif name == "turned":
        s.lights[1].up = (1.0, 0.3, 0.1)
        s.lights[2].up = (-0.2, 0.9, 0.4)
    elif name == "washer alone, dark":
        s.lights = [s.lights[2]]
        s.lights[0].profile = 1
        s.env_strength = 0.0
    return s


@pytest.mark.parametrize("name", ["far washer", "turned", "washer alone, dark"])
def test_variants_have_the_oracle_bits(rtg, oracle_lib, name):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(variant(name))
    f = rtg.Scene(rsb).film()
    f.render(0, 4)
    rgb, w, al, l2, _ = oracle_lib.OracleScene(rsb).render_film(0, 4, threads=8)
    for a, b in zip(f.read(), (rgb, w, al, l2)):
        assert np.array_equal(np.asarray(a).view(np.uint32), b.view(np.uint32))


def test_paths_match_the_oracle(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(l5())
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    rng = np.random.default_rng(13)
    n = 5000
    xys = np.stack([rng.integers(0, g.width, n), rng.integers(0, g.height, n), rng.integers(0, 256, n)], 1).astype(np.uint32)
    got, want = g.render_paths(xys), o.paths(xys)
    assert np.allclose(got[:, :4], want[:, :4], rtol=1.0e-4, atol=1.0e-6)
    exact = np.mean(np.all(got[:, :4].view(np.uint32) == want[:, :4].view(np.uint32), axis=1))
    print(f"L5: {exact * 100:.2f}% of paths bit-exact")
