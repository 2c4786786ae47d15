"""rtg_render_progressive_noalloc, the allocation-free progressive render, through the C ABI.

It runs the wavefront with its path state in the library's fixed device array instead of
per-scene buffers. Its films are compared with those of rtg_render_progressive on the same
scene and samples, within the path tolerance (relative 1e-4; the two are built to agree to the
bit), after each of two calls in a row. The file's name makes pytest collect it last; it also
passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1.0e-4, 1.0e-6


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def film_sums(film):
    return [np.array(a) for a in film.read()]


def assert_films_agree(a, b):
    for x, y in zip(film_sums(a), film_sums(b)):
        assert np.allclose(x, y, rtol=RTOL, atol=ATOL)


def test_two_calls_in_a_row_match_the_progressive_render(rtg, example_rsb, pins):
    # 512 x 384 pixels: three bands of 128 rows, each a wave of 65,536 paths.
    s = rtg.Scene(example_rsb)
    ref, fixed = s.film(), s.film()
    for first, count in ((0, 2), (2, 2)):
        rays_ref = ref.render(first, count)
        rays_fixed = fixed.render_noalloc(first, count)
        assert rays_fixed == rays_ref
        assert_films_agree(fixed, ref)
    # Four samples in all: the reference's pinned film hash.
    assert rtg.fnv1a(fixed.resolve()) == pins["film_hashes"]["example_4spp"]


def test_waves_of_several_samples(rtg, small_product_rsb):
    # 96 x 64 pixels: 16 samples run as waves of 10 and 6 samples; two calls in a row.
    s = rtg.Scene(small_product_rsb)
    ref, fixed = s.film(), s.film()
    for first in (0, 16):
        ref.render(first, 16)
        fixed.render_noalloc(first, 16)
        assert_films_agree(fixed, ref)


def test_handles_and_empty_work(rtg, cfg0_rsb):
    L = rtg.lib()
    s = rtg.Scene(cfg0_rsb)
    f = s.film()
    rays = ctypes.c_uint64(7)
    assert L.rtg_render_progressive_noalloc(0, f.handle, 0, 1, ctypes.byref(rays)) == rtg.STATUS_BAD_HANDLE
    assert L.rtg_render_progressive_noalloc(s.handle, 0, 0, 1, ctypes.byref(rays)) == rtg.STATUS_BAD_FILM
    assert L.rtg_render_progressive_noalloc(s.handle, f.handle, 0, 0, ctypes.byref(rays)) == rtg.STATUS_OK
    assert rays.value == 0
    assert float(film_sums(f)[1].sum()) == 0.0
    # A film over part of the image, partly outside it.
    g = rtg.Film(s, 200, 100, 100, 50)
    ref = rtg.Film(s, 200, 100, 100, 50)
    g.render_noalloc(3, 2)
    ref.render(3, 2)
    assert_films_agree(g, ref)


def test_fused_guides_match_the_progressive_render(rtg, example_rsb):
    # A film with fused guides takes each render's first-hit albedo into its guide sums; the
    # allocation-free render fills them from its own array. The denoised image reads those sums,
    # so it agrees only when both renders added the same albedo.
    s = rtg.Scene(example_rsb)
    ref, fixed = s.film(), s.film()
    ref.fuse_guides(True)
    fixed.fuse_guides(True)
    for first, count in ((0, 2), (2, 2)):
        ref.render(first, count)
        fixed.render_noalloc(first, count)
        assert_films_agree(fixed, ref)
    assert np.allclose(fixed.denoise(4), ref.denoise(4), rtol=RTOL, atol=ATOL)
