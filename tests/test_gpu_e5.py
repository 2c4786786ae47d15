"""The E5 features on the GPU, through the C ABI: an HDRI environment (RGBE bitmap, 2-D importance
sampling, rotation), a background image, cut-outs (paths pass them without a vertex, in extra
rounds of the wave) and thin walls, and shadow rays that walk through both.

* The E5 scene at 4 samples has the reference's pinned film hash (render.rs:1086-1107), under its
  HDRI and under the classic sky; other skies (low and high suns, turbidity, a sun below the
  horizon) have the oracle's film bits.
* Variants (background image fill, fit and stretch over a sub-rectangle; an 8-bit sRGB HDRI; the
  cut-out card alone; the thin card alone; a clamp on indirect light) have the oracle's film bits.
* Per-path radiance equals the oracle's within 1e-4 (reported bit-exact share).
* The batched queue renders E5 variants with the bits of the plain path; a scene update without
  BMAP sections keeps the loaded bitmaps; the adjoint refuses scenes with passable surfaces.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def e5(**changes):
    from repackshot_b200 import scenes
    s = scenes.e5_scene()
    for k, v in changes.items():
        setattr(s, k, v)
    return s


def bits_equal_oracle(rtg, oracle_lib, rsb, count=4):
    g = rtg.Scene(rsb)
    f = g.film()
    f.render(0, count)
    rgb, w, al, l2, _ = oracle_lib.OracleScene(rsb).render_film(0, count, threads=8)
    return all(np.array_equal(np.asarray(a).view(np.uint32), b.view(np.uint32)) for a, b in zip(f.read(), (rgb, w, al, l2)))


def test_e5_has_the_pinned_hash(rtg, pins):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.e5_scene()))
    f = s.film()
    f.render(0, 1)
    f.render(1, 3)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["e5_hdri_4spp"]
    g = s.film()
    g.render_noalloc(0, 4)
    assert rtg.fnv1a(g.resolve()) == pins["film_hashes"]["e5_hdri_4spp"]


def test_e5_under_the_classic_sky_has_the_pinned_hash(rtg, pins):
    from repackshot_b200 import scenes
    f = rtg.Scene(scenes.to_rsb(scenes.e5_scene(sky=True))).film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["e5_sky_4spp"]


def test_e5c_under_the_physical_sky_has_the_pinned_hash(rtg, pins):
    # render.rs:1112-1128: the physical sky tabulated on the host, sampled and seen on the device.
    from repackshot_b200 import scenes
    f = rtg.Scene(scenes.to_rsb(scenes.e5c_scene())).film()
    f.render(0, 2)
    f.render(2, 2)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["e5c_physical_sky_4spp"]


def sky(**changes):
    from repackshot_b200 import scenes
    s = scenes.e5_scene(sky=True)
    for k, v in changes.items():
        setattr(s, k, v)
    return s


SKIES = {"low sun, hazy": dict(sun_elevation_deg=5.0, sky_turbidity=8.0), "high sun, clear": dict(sun_elevation_deg=80.0,
                                                                                                   sky_turbidity=1.0),
         "below the horizon, clamped": dict(sun_elevation_deg=-10.0, sun_azimuth_deg=200.0, env_strength=2.0),
         "sky as background image": dict(background_mode=3)}


@pytest.mark.parametrize("name", list(SKIES))
def test_skies_have_the_oracle_bits(rtg, oracle_lib, name):
    from repackshot_b200 import scenes
    assert bits_equal_oracle(rtg, oracle_lib, scenes.to_rsb(sky(**SKIES[name])))


def variants():
    from repackshot_b200 import scenes
    out = {}
    out["fit, sub-rectangle"] = e5(backplate_fit=1, backplate_rect=(0.1, 0.2, 0.9, 0.7))
    out["stretch"] = e5(backplate_fit=2)
    out["fill, wide frame"] = e5(width=200, height=60)
    srgb = e5()
    w, h = 32, 16
    px = bytes((x * 8 + y * 3) % 256 for y in range(h) for x in range(w) for _ in range(3))
    srgb.bitmaps = [scenes.Bitmap(0, w, h, px), srgb.bitmaps[1]]
    srgb.env_rotation = -75.0
    out["8-bit HDRI"] = srgb
    cut = e5()
    cut.instances = [i for i in cut.instances if i.material_id != 3]
    out["cut-out card only"] = cut
    thin = e5()
    thin.instances = [i for i in thin.instances if i.material_id != 4]
    out["thin card only"] = thin
    out["clamped"] = e5(clamp_indirect=0.5)
    out["no map, dome"] = e5(hdri_map=0xFFFFFFFF)
    return out


@pytest.mark.parametrize("name", list(variants()))
def test_variants_have_the_oracle_bits(rtg, oracle_lib, name):
    from repackshot_b200 import scenes
    assert bits_equal_oracle(rtg, oracle_lib, scenes.to_rsb(variants()[name]))


def test_paths_match_the_oracle(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.e5_scene())
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    rng = np.random.default_rng(9)
    n = 6000
    xys = np.stack([rng.integers(0, g.width, n), rng.integers(0, g.height, n), rng.integers(0, 256, n)], 1).astype(np.uint32)
    got, want = g.render_paths(xys), o.paths(xys)
    assert np.allclose(got[:, :4], want[:, :4], rtol=1.0e-4, atol=1.0e-6)
    exact = np.mean(np.all(got[:, :4].view(np.uint32) == want[:, :4].view(np.uint32), axis=1))
    print(f"E5: {exact * 100:.2f}% of paths bit-exact")


def test_queue_of_e5_variants_matches_the_plain_path(rtg):
    from repackshot_b200 import scenes
    base = scenes.e5_scene()
    scene = rtg.Scene(scenes.to_rsb(base))
    jobs = []
    for k in range(3):
        v = copy.deepcopy(base)
        v.lights[0].power *= 1.0 + 0.5 * k
        v.materials[4].opacity = 0.2 + 0.3 * k
        v.env_rotation = 30.0 + 40.0 * k
        v.width, v.height = [(160, 120), (96, 64), (120, 90)][k]
        jobs.append(v)
    for graph in (False, True):
        q = rtg.Queue(scene)
        # job files without meshes or bitmaps keep the scene's
        films = [q.add(scenes.to_rsb(_without_bitmaps(v), meshes=False), 0, 3, v.width, v.height) for v in jobs]
        q.run(graph=graph)
        for f, v in zip(films, jobs):
            plain = rtg.Scene(scenes.to_rsb(v)).film()
            plain.render(0, 3)
            for a, b in zip(f.read(), plain.read()):
                assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def _without_bitmaps(v):
    w = copy.deepcopy(v)
    w.bitmaps = []
    return w


def test_update_without_bitmaps_keeps_them(rtg, pins):
    from repackshot_b200 import scenes
    base = scenes.e5_scene()
    s = rtg.Scene(scenes.to_rsb(base))
    moved = _without_bitmaps(base)
    moved.lights[0].power *= 2.0
    s.update(scenes.to_rsb(moved, meshes=False))
    s.update(scenes.to_rsb(_without_bitmaps(base), meshes=False))
    f = s.film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["e5_hdri_4spp"]


def test_adjoint_refuses_passable_surfaces(rtg):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.e5_scene()))
    nm, nl = s.adjoint_params()
    with pytest.raises(rtg.RtgError) as e:
        s.adjoint(s.film(), np.zeros((s.height, s.width, 3), np.float32), 0, 2)
    assert e.value.status == rtg.STATUS_BAD_SCENE and "cut-outs" in str(e.value)
