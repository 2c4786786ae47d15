"""The section view (Q1) on the GPU (engine/crates/rt-core/src/geometry/section.rs,
render/section_tests.rs). The Q1 fixture is the E5 scene cut in two by the plane x = 0 with a cap: a
glass sphere halved, its cap shaded as the glass; the floor exempt from the section.

* the film at 4 spp has the reference's pinned hash, and the same file without its section, or with a
  plane that cuts nothing, keeps E5's pinned hash;
* nearest hits (instance, triangle or the cap, t bits) and any-hit answers of random rays through the
  cut are the oracle's, bit for bit, for camera and other rays;
* the exact passes see the cap as the cut solid (its instance and the plane's normal);
* the adjoint and the batched queue refuse a scene with a section.
"""
import struct
from pathlib import Path

import numpy as np
import pytest

from rays import random_rays
from test_oracle_section import with_section

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
CAP = 0xFFFFFFFF


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def q1() -> bytes:
    return (GOLDEN / "q1.rsb").read_bytes()


def film_hash(rtg, rsb: bytes) -> int:
    f = rtg.Scene(rsb).film()
    f.render(0, 4)
    return rtg.fnv1a(f.resolve())


def test_q1_has_the_pinned_hash(rtg, pins):
    assert film_hash(rtg, q1()) == pins["film_hashes"]["q1_section_4spp"]


@pytest.mark.parametrize("payload", [None, struct.pack("<I4f", 1, 0.0, 0.0, 1.0, 1.0e5)], ids=["no section", "far plane"])
def test_a_section_that_cuts_nothing_is_the_scene_of_before(rtg, pins, payload):
    assert film_hash(rtg, with_section(q1(), payload)) == pins["film_hashes"]["e5_hdri_4spp"]


@pytest.mark.parametrize("cap", [1, 0], ids=["capped", "open cut"])
def test_queries_through_the_cut_are_the_oracles(rtg, oracle_lib, cap):
    rsb = with_section(q1(), struct.pack("<I4f", cap, 1.0, 0.0, 0.0, 0.0))
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    rays = random_rays(40000, (-500, -400, 0), (400, 300, 300), seed=31)
    rays[::4, 7] = np.float32(250.0)  # bounded intervals: rays that end before or after the plane
    for camera in (False, True):
        want, _ = o.trace(rays, camera=camera)
        got = g.trace(rays, camera=camera)
        assert np.array_equal(got, want)
    if cap:
        assert (want[:, 1] == CAP).sum() > 100, "rays hit the cap"
    assert np.array_equal(g.trace(rays, any_hit=True).astype(np.uint8), o.occluded(rays))


def test_the_passes_see_the_cap_as_the_cut_solid(rtg, oracle_lib):
    g, o = rtg.Scene(q1()), oracle_lib.OracleScene(q1())
    w, h = g.width, g.height
    st, words = rtg.tile_passes(g.handle, 0, 0, w, h, 0x3E)
    assert st == rtg.STATUS_OK
    n = w * h
    normal, depth, part, material = o.passes()
    assert np.array_equal(words[:3 * n], np.ascontiguousarray(normal, np.float32).view(np.uint32).reshape(-1))
    assert np.array_equal(words[3 * n:4 * n], np.ascontiguousarray(depth, np.float32).view(np.uint32).reshape(-1))
    assert np.array_equal(words[4 * n:5 * n], part.reshape(-1))
    assert np.array_equal(words[5 * n:6 * n], material.reshape(-1))
    # section_tests.rs:45-92: the glass sphere (instance 0, id 1 in the pass; 0 is the background) is
    # seen cut, its cap facing the camera on the removed side with the plane's normal +x, material 1.
    nx = normal.reshape(-1, 3)
    on_cap = (part.reshape(-1) == 1) & (np.abs(nx[:, 0] - 1.0) < 1e-5) & (np.abs(nx[:, 1]) < 1e-5) & (np.abs(nx[:, 2]) < 1e-5)
    assert on_cap.sum() > 500
    assert (material.reshape(-1)[on_cap] == 1).all()
    for sample in (0, 3):
        st, alb = rtg.tile_albedo(g.handle, 0, 0, w, h, sample)
        assert st == rtg.STATUS_OK
        assert np.array_equal(np.ascontiguousarray(alb, np.float32).view(np.uint32),
                              np.ascontiguousarray(o.albedo(sample), np.float32).view(np.uint32).reshape(-1))


def test_the_adjoint_and_the_queue_refuse_a_section(rtg):
    s = rtg.Scene(q1())
    with pytest.raises(rtg.RtgError, match="unsupported"):
        s.adjoint(s.film(), np.zeros((s.height, s.width, 3), np.float32), 0, 1)
    q = rtg.Queue(s)
    with pytest.raises(rtg.RtgError, match="a section view"):
        q.add(strip_meshes(q1()), 0, 1, s.width, s.height)


def strip_meshes(rsb: bytes) -> bytes:
    """The file without its MESH sections: a queue job keeps the scene's geometry."""
    from repackshot_b200.__main__ import _sections
    out = rsb[:8 + struct.unpack_from("<I", rsb, 4)[0]]
    for tag, start, at, n in _sections(rsb):
        if tag != b"MESH":
            out += rsb[start:at + n]
    return out


# ---- the synthetic scene of every rule (repackshot_b200.scenes.section_scene) ---------------------

def test_every_rule_is_the_oracles(rtg, oracle_lib):
    """Welded, rotated and scaled, inward, open, thin and camera-hidden solids, the studio floor and
    the studio box behind 60 slices: nearest hits, any-hit answers, the exact passes and a 4-spp film
    are the oracle's bit for bit."""
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.section_scene())
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    rays = np.concatenate([random_rays(60000, (-250, -400, 5), (250, 400, 150), seed=41),
                           random_rays(20000, (200, -100, 0), (320, 100, 150), seed=42)])
    rays[::5, 7] = np.float32(120.0)
    for camera in (False, True):
        want, _ = o.trace(rays, camera=camera)
        assert np.array_equal(g.trace(rays, camera=camera), want)
    assert (want[:, 1] == CAP).sum() > 500
    assert np.array_equal(g.trace(rays, any_hit=True).astype(np.uint8), o.occluded(rays))
    w, h = g.width, g.height
    st, words = rtg.tile_passes(g.handle, 0, 0, w, h, 0x3E)
    assert st == rtg.STATUS_OK
    normal, depth, part, material = o.passes()
    n = w * h
    assert np.array_equal(words[:3 * n], np.ascontiguousarray(normal, np.float32).view(np.uint32).reshape(-1))
    assert np.array_equal(words[4 * n:5 * n], part.reshape(-1))
    f = g.film()
    f.render(0, 4)
    rgb, wt, _, _, _ = o.render_film(0, 4, threads=16)
    assert rtg.fnv1a(f.resolve()) == oracle_lib.fnv1a(oracle_lib.resolve(rgb, wt))


def test_an_update_brings_and_takes_the_section(rtg, pins):
    """rt_scene_update (ffi.rs:68-88, rsb.rs: an update replaces the section; a file without SECT has
    none): E5 updated with Q1's file without its meshes renders Q1, and back to E5."""
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.e5_scene()))

    def film():
        f = s.film()
        f.render(0, 4)
        return rtg.fnv1a(f.resolve())

    assert film() == pins["film_hashes"]["e5_hdri_4spp"]
    s.update(strip_meshes(q1()))
    assert film() == pins["film_hashes"]["q1_section_4spp"]
    s.update(strip_meshes(scenes.to_rsb(scenes.e5_scene())))
    assert film() == pins["film_hashes"]["e5_hdri_4spp"]
    s.update(strip_meshes(with_section(q1(), None)))
    assert film() == pins["film_hashes"]["e5_hdri_4spp"]
