"""The oracle's pixel filters and edge samples against the reference's known answers
(engine/crates/rt-core/src/pixel_filter.rs and its tests, render.rs:1224-1250):

* the Blackman-Harris inverse CDF, generated here by bisection of the window's integral, has the
  bytes of the reference's table (SHA-256 pinned from pixel_filter.rs:64);
* the standard filter is the uniform position itself, none the centre, the tent and
  Blackman-Harris stay inside their widths and start at their edges;
* the E11 scene (the example with Blackman-Harris and two samples per index on its edges) has the
  reference's pinned 4-sample hash, for 32- and 23-pixel tiles, and with the standard filter and no
  edge samples it is the example's pinned film again.
"""
import hashlib

import numpy as np

from repackshot_b200 import scenes


def test_blackman_harris_table_is_the_reference_table(oracle_lib, pins):
    t = oracle_lib.blackman_harris_table()
    assert len(t) == pins["blackman_harris_inv_cdf"]["count"]
    assert hashlib.sha256(t.astype("<f4").tobytes()).hexdigest() == pins["blackman_harris_inv_cdf"]["sha256"]
    assert t[0] == -1.5 and np.all(np.diff(t) > 0) and np.array_equal(t, -t[::-1])


def test_filter_offsets(oracle_lib):
    rng = np.random.default_rng(7)
    u = rng.random(10_000, dtype=np.float32)
    assert np.array_equal(oracle_lib.filter_offset(0, u).view(np.uint32), u.view(np.uint32))
    assert np.array_equal(oracle_lib.filter_offset(99, u).view(np.uint32), u.view(np.uint32))
    assert np.all(oracle_lib.filter_offset(1, u) == 0.5)
    soft = oracle_lib.filter_offset(2, u)
    fine = oracle_lib.filter_offset(3, u)
    assert np.all((soft >= -0.5) & (soft <= 1.5)) and np.all((fine >= -1.0) & (fine <= 2.0))
    ends = np.array([0.0], np.float32)
    assert oracle_lib.filter_offset(2, ends)[0] == -0.5 and oracle_lib.filter_offset(3, ends)[0] == -1.0


def test_e11_has_the_pinned_hash_for_any_tile_cut(oracle_lib, pins):
    o = oracle_lib.OracleScene(scenes.to_rsb(scenes.e11_scene()))
    for tile in (32, 23):
        rgb, w, _, _, _ = o.render_film(0, 4, tile=tile, threads=8)
        assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["e11_edges_4spp"]
    edges = o.edge_mask()
    assert 0 < int(edges.sum()) < edges.size // 2


def test_without_edges_and_filter_it_is_the_example(oracle_lib, pins):
    s = scenes.e11_scene()
    s.pixel_filter, s.edge_supersample = 0, 1
    o = oracle_lib.OracleScene(scenes.to_rsb(s))
    rgb, w, _, _, _ = o.render_film(0, 4, threads=8)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["example_4spp"]
    assert int(o.edge_mask().sum()) == 0
