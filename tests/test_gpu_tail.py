"""The tail kernel (k_tail: a wave's last rounds in one launch, a path per thread) across the
path's features. With the tail limit at 2^20 every path of these small scenes runs through k_tail
from the wave's third round on, so each of its vertices is shaded there and its shadow ray traced
there. The reference's pinned film hashes (render.rs:1036-1128, render/k3_tests.rs:17-22) still
hold: the example, E5 under its HDRI, the classic and the physical sky, and the panoramic K3 views
(the plan has a thin pane, so it keeps the wavefront: a scene with passable surfaces never takes the
tail). Scenes without pins (every light kind at once; emissive meshes sampled as lights) give the
same film, bit for bit, with the tail at 2^20 and off.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
ALL_IN_TAIL = 1 << 20


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def pinned_cases():
    from repackshot_b200 import scenes
    return {
        "example_4spp": lambda: scenes.to_rsb(scenes.example_scene()),
        "e5_hdri_4spp": lambda: scenes.to_rsb(scenes.e5_scene()),
        "e5_sky_4spp": lambda: scenes.to_rsb(scenes.e5_scene(sky=True)),
        "e5c_physical_sky_4spp": lambda: scenes.to_rsb(scenes.e5c_scene()),
        "k3_panorama_4spp": lambda: (GOLDEN / "k3-panorama.rsb").read_bytes(),
        "k3_fisheye_4spp": lambda: (GOLDEN / "k3-fisheye.rsb").read_bytes(),
        "k3_plan_4spp": lambda: (GOLDEN / "k3-plan.rsb").read_bytes(),
    }


@pytest.mark.parametrize("name", sorted(pinned_cases()))
def test_pinned_scenes_keep_their_hashes_in_the_tail(rtg, pins, name):
    s = rtg.Scene(pinned_cases()[name]())
    s.set_tuning(tail_paths=ALL_IN_TAIL)
    assert s.tuning()["tail_paths"] == ALL_IN_TAIL
    f = s.film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"][name]


@pytest.mark.parametrize("which", ["light kinds", "emissive meshes"])
def test_scenes_without_pins_render_the_same_film_in_the_tail(rtg, which):
    from repackshot_b200 import scenes
    desc = scenes.light_kinds_scene(128, 96) if which == "light kinds" else scenes.emissive_scene()
    s = rtg.Scene(scenes.to_rsb(desc))
    films = []
    for tail in (0, ALL_IN_TAIL):
        s.set_tuning(tail_paths=tail)
        f = s.film()
        f.render(0, 3)
        f.render(3, 5)
        films.append([np.asarray(a).view(np.uint32).copy() for a in f.read()])
    for a, b in zip(*films):
        assert np.array_equal(a, b)
