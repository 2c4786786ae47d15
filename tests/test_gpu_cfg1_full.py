"""Parity on the 1080p product scene at its full size: the geometry the benchmark renders.

The scene is the benchmark's own: 1920 x 1080, 64 spp, depth 12, the seeded (2,3) torus knot of
1024 x 512 segments (1,048,576 triangles) in 16 materials (GGX conductors, rough dielectrics,
Lambert), three softboxes and a gradient dome. Against the oracle on identical inputs:

* traversal: nearest hits (instance, triangle, t bits) of 20,000 incoherent rays and about
  20,000 surface rays (leaving hit points of the knot) bit-exact, both ray classes; the first 2,000 also against brute force over every
  triangle; any-hit flags bit-exact;
* paths: 4,000 per-path radiances of random (pixel, sample) pairs within 1e-4 relative;
* film: four row bands of 1920 x 8 pixels at the frame's 64 spp within rel-MSE 1e-3 (rel-MSE =
  mean of (a - b)^2 / (b^2 + 1e-2) over pixels and channels).
"""
import os

import numpy as np
import pytest

from rays import random_rays, surface_rays

pytestmark = pytest.mark.gpu

WIDTH, HEIGHT, SPP, DEPTH = 1920, 1080, 64, 12
PATH_RTOL = 1.0e-4
REL_MSE_MAX = 1.0e-3
BOX = ((-1500, -1500, 0), (1500, 1500, 2500))


def rel_mse(a, b, eps=1.0e-2):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.mean((a - b) ** 2 / (b * b + eps)))


@pytest.fixture(scope="module")
def pair(oracle_lib):
    import repackshot_b200 as rtg
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.product_scene(width=WIDTH, height=HEIGHT, spp=SPP, depth=DEPTH))
    g = rtg.Scene(rsb)
    assert g.triangles >= 1_048_576
    return rtg, g, oracle_lib.OracleScene(rsb)


def test_full_knot_nearest_hits_are_bit_exact(pair):
    _, g, o = pair
    rays = np.concatenate([random_rays(20000, *BOX, seed=31), surface_rays(o, 13000, seed=32)])
    assert len(rays) >= 35000
    for camera in (False, True):
        got = g.trace(rays, camera=camera)
        want, _ = o.trace(rays, camera=camera)
        assert np.array_equal(got, want)
        brute, _ = o.trace(rays[:2000], camera=camera, brute=True)
        assert np.array_equal(got[:2000], brute)
    hit = np.mean(got[:, 0] != 0xFFFFFFFF)
    print(f"full knot: {len(rays)} rays, {hit * 100:.1f}% hit")


def test_full_knot_any_hits_are_bit_exact(pair):
    _, g, o = pair
    rays = np.concatenate([random_rays(20000, *BOX, seed=33), surface_rays(o, 10000, seed=34)])
    rays[::3, 7] = np.float32(300.0)  # bounded shadow-ray intervals
    assert np.array_equal(g.trace(rays, any_hit=True).astype(np.uint8), o.occluded(rays))


def test_full_knot_path_radiance_matches(pair):
    _, g, o = pair
    rng = np.random.default_rng(35)
    n = 4000
    xys = np.stack([rng.integers(0, WIDTH, n), rng.integers(0, HEIGHT, n), rng.integers(0, SPP, n)], 1).astype(np.uint32)
    got, want = g.render_paths(xys), o.paths(xys)
    assert np.allclose(got[:, :4], want[:, :4], rtol=PATH_RTOL, atol=1e-6)
    exact = np.mean(np.all(got[:, :4].view(np.uint32) == want[:, :4].view(np.uint32), axis=1))
    print(f"full knot: {exact * 100:.2f}% of 4000 paths bit-exact")


def test_full_frame_bands_at_64_spp_within_rel_mse(pair, oracle_lib):
    rtg, g, o = pair
    for y in (60, 390, 700, 1010):
        band = rtg.Film(g, 0, y, WIDTH, 8)
        band.render(0, SPP)
        got = band.resolve()
        rgb, w, _, _, _ = o.render_film(0, SPP, x=0, y=y, w=WIDTH, h=8, threads=os.cpu_count() or 1)
        want = oracle_lib.resolve(rgb, w)
        err = rel_mse(got, want)
        exact = np.mean(got.view(np.uint32) == want.view(np.uint32))
        print(f"rows {y}-{y + 7} at 64 spp: rel-MSE {err:.3e}, bit-exact values {exact * 100:.3f}%")
        assert err <= REL_MSE_MAX
