"""Pixel filters and edge samples (E11) on the GPU, through the C ABI.

* The E11 scene (the example with the Blackman-Harris filter and two samples per sample index on
  its edges) has the reference's pinned 4-sample film hash (render.rs:1224-1250), rendered in one
  call or several, with waves small enough to split the edge pixels and the sample indices.
* Other filters and edge factors (tent, none, k = 3 and 16), edges in the E5 scene (cut-outs, an
  HDRI), a film over part of the image and single-sample tiles have the oracle's bits.
* Calls that cannot take edge samples refuse them: the batched queue, the adjoint and the
  allocation-free render.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def test_e11_has_the_pinned_hash(rtg, pins):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.e11_scene()))
    f = s.film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["e11_edges_4spp"]
    g = s.film()
    g.render(0, 1)
    g.render(1, 3)
    assert rtg.fnv1a(g.resolve()) == pins["film_hashes"]["e11_edges_4spp"]
    s.set_path_capacity(5000)  # splits the rows, the edge pixels and the sample indices
    h = s.film()
    h.render(0, 4)
    assert rtg.fnv1a(h.resolve()) == pins["film_hashes"]["e11_edges_4spp"]


def variant(name):
    from repackshot_b200 import scenes
    if name.startswith("e5"):
        s = scenes.e5_scene()
        s.pixel_filter, s.edge_supersample = 3, 3
        return s
    s = scenes.example_scene()
    s.width, s.height = 160, 120
    s.pixel_filter, s.edge_supersample = {"tent, k 3": (2, 3), "none, k 16": (1, 16), "standard, k 2": (0, 2),
                                          "Blackman-Harris, k 1": (3, 1)}[name]
    return s


@pytest.mark.parametrize("name", ["tent, k 3", "none, k 16", "standard, k 2", "Blackman-Harris, k 1", "e5, k 3"])
def test_variants_have_the_oracle_bits(rtg, oracle_lib, name):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(variant(name))
    f = rtg.Scene(rsb).film()
    f.render(0, 3)
    rgb, w, al, l2, _ = oracle_lib.OracleScene(rsb).render_film(0, 3, threads=8)
    for a, b in zip(f.read(), (rgb, w, al, l2)):
        assert np.array_equal(np.asarray(a).view(np.uint32), b.view(np.uint32))


def test_part_of_the_image_and_tiles(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.e11_scene())
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    f = rtg.Film(g, 200, 100, 150, 120)
    f.render(2, 2)
    rgb, w, al, l2, _ = o.render_film(2, 2, 200, 100, 150, 120)
    for a, b in zip(f.read(), (rgb, w, al, l2)):
        assert np.array_equal(np.asarray(a).view(np.uint32), b.view(np.uint32))
    for (x, y) in [(240, 176), (0, 0), (500, 370)]:
        got = g.render_tile(x, y, 32, 32, 3, rgba=True)
        want = o.render_tile(x, y, 32, 32, 3, rgba=True)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_calls_without_edge_samples_refuse_them(rtg):
    from repackshot_b200 import scenes
    e11 = scenes.e11_scene()
    s = rtg.Scene(scenes.to_rsb(e11))
    with pytest.raises(rtg.RtgError) as e:
        s.film().render_noalloc(0, 1)
    assert e.value.status == rtg.STATUS_BAD_SCENE
    with pytest.raises(rtg.RtgError) as e:
        s.adjoint(s.film(), np.zeros((s.height, s.width, 3), np.float32), 0, 2)
    assert e.value.status == rtg.STATUS_BAD_SCENE
    q = rtg.Queue(rtg.Scene(scenes.to_rsb(scenes.example_scene())))
    with pytest.raises(rtg.RtgError) as e:
        q.add(scenes.to_rsb(e11, meshes=False), 0, 1, e11.width, e11.height)
    assert e.value.status == rtg.STATUS_BAD_SCENE
