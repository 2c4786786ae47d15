"""The guide passes and the denoiser (engine/crates/rt-post/src/denoise.rs) on the GPU, through the
C ABI, against the oracle and the reference's pinned hashes (denoise/tests.rs:369-528):

* rtg_render_tile_passes and rtg_render_tile_albedo give the oracle's bits (the example; E11 with
  its edge sub-samples);
* rtg_denoise_with on the oracle's input words gives the oracle's bits and the pinned hashes of the
  denoised example (the full filter at 4 samples, the viewport's at 2 and 4), bands of rows give
  those rows of the whole image, strength 0 and 0.5 blend as the reference does;
* the whole path on the device (rtg_render_progressive, rtg_film_guides, rtg_film_denoise) gives
  the pinned hash;
* random planes with fireflies next to each other (the clamp's raster-order dependence), too few
  samples (the spatial variance), non-finite guides and several parts give the oracle's bits.
"""
import numpy as np
import pytest

from denoise_cases import example_input, fnv1a_floats, means, rgba_sums

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


@pytest.fixture(scope="module")
def example4(oracle_lib):
    return example_input(oracle_lib, 4)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_passes_and_albedo_are_the_oracle_ones(rtg, oracle_lib):
    from repackshot_b200 import scenes
    for s in (scenes.example_scene(), scenes.e11_scene()):
        s.width, s.height = 160, 120
        rsb = scenes.to_rsb(s)
        sc, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
        st, words = rtg.tile_passes(sc.handle, 0, 0, 160, 120, 0x3E)
        assert st == rtg.STATUS_OK
        n = 160 * 120
        normal, depth, part, material = o.passes()
        assert np.array_equal(words[:3 * n], bits(normal).reshape(-1))
        assert np.array_equal(words[3 * n:4 * n], bits(depth).reshape(-1))
        assert np.array_equal(words[4 * n:5 * n], part.reshape(-1)) and np.array_equal(words[5 * n:6 * n], material.reshape(-1))
        # the circle of confusion (passes.rs:130) from the depth and the camera, in float32
        f32 = np.float32
        aperture = f32(s.focal_mm) / f32(s.fstop)
        with np.errstate(invalid="ignore", divide="ignore"):
            on_plane = (aperture * np.abs(depth - f32(s.focus_dist))).astype(f32) / depth
        pixel = (f32(s.sensor_mm) / f32(160)) * (f32(s.focus_dist) / f32(s.focal_mm))
        coc = np.where((depth > 0) & np.isfinite(depth), (on_plane / pixel).astype(f32), f32(0)).astype(f32)
        assert np.array_equal(words[6 * n:], bits(coc).reshape(-1))
        st, sub = rtg.tile_passes(sc.handle, 150, 110, 20, 20, 0x08)  # partly outside the image
        assert st == rtg.STATUS_OK and sub.reshape(20, 20)[10:, :].max() == 0
        for sample in (0, 3):
            st, alb = rtg.tile_albedo(sc.handle, 0, 0, 160, 120, sample)
            assert st == rtg.STATUS_OK and np.array_equal(bits(alb), bits(o.albedo(sample)).reshape(-1))


def test_the_denoised_example_is_the_oracle_image_and_has_the_pinned_hash(rtg, oracle_lib, example4, pins):
    o, words, _, _ = example4
    out = rtg.denoise(words, o.width, o.height, 4)
    assert np.array_equal(bits(out), bits(oracle_lib.denoise(words, o.width, o.height, 4)))
    assert fnv1a_floats(means(out, 4)) == pins["denoised"]["example_4spp"]
    assert fnv1a_floats(means(rtg.denoise(words, o.width, o.height, 4, preset=1), 4)) == pins["denoised"]["viewport_example_4spp"]
    o2, words2, _, _ = example_input(oracle_lib, 2)
    out2 = rtg.denoise(words2, o2.width, o2.height, 2, preset=1)
    assert fnv1a_floats(means(out2, 2)) == pins["denoised"]["viewport_example_2spp"]
    assert np.array_equal(bits(rtg.denoise(words2, o2.width, o2.height, 2)), bits(oracle_lib.denoise(words2, o2.width, o2.height, 2)))


def test_bands_strength_and_refusals(rtg, oracle_lib, example4):
    from test_oracle_denoise import band_words
    o, words, _, _ = example4
    w, h = o.width, o.height
    whole = rtg.denoise(words, w, h, 4)
    halo = rtg.lib().rtg_denoise_halo(0)
    assert (halo, rtg.lib().rtg_denoise_halo(1), rtg.lib().rtg_denoise_halo(5)) == (72, 24, 0)
    parts = []
    for k in range(3):
        y0, y1 = h * k // 3, h * (k + 1) // 3
        lo, hi = max(0, y0 - halo), min(h, y1 + halo)
        parts.append(rtg.denoise(band_words(words, w, h, lo, hi), w, h, 4, origin_y=lo, rows=hi - lo, y0=y0, y1=y1))
    assert np.array_equal(bits(np.concatenate(parts)), bits(whole))
    for s in (0.0, 0.5, 0.25):
        assert np.array_equal(bits(rtg.denoise(words, w, h, 4, strength=s)), bits(oracle_lib.denoise(words, w, h, 4, strength=s)))
    with pytest.raises(rtg.RtgError):
        rtg.denoise(band_words(words, w, h, 100, 200), w, h, 4, origin_y=100, rows=100, y0=120, y1=180)
    with pytest.raises(rtg.RtgError):
        rtg.denoise(words, w, h, 4, preset=3)


def test_the_device_path_has_the_pinned_hash(rtg, pins):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.example_scene()))
    f = s.film()
    f.render(0, 4)
    f.guides(0, 4)
    out = f.denoise(4)
    assert fnv1a_floats(means(out, 4)) == pins["denoised"]["example_4spp"]
    g = s.film()  # the guides in two calls, the albedo summed in sample order
    g.render(0, 4)
    g.guides(0, 1)
    g.guides(1, 3)
    assert np.array_equal(bits(g.denoise(4)), bits(out))
    half = f.denoise(4, strength=0.5)
    rgb, _, alpha, _ = f.read()
    noisy = rgba_sums(rgb, alpha).reshape(out.shape)
    want = (noisy[..., :3] * np.float32(0.5) + out[..., :3] * np.float32(0.5)).astype(np.float32)
    assert np.array_equal(bits(half[..., :3]), bits(want))


@pytest.mark.parametrize("seed, samples", [(1, 8), (2, 2), (3, 1), (4, 16)])
def test_random_planes_are_the_oracle_image(rtg, oracle_lib, seed, samples):
    rng = np.random.default_rng(seed)
    w, h = 97, 61
    n = w * h
    part = (rng.integers(0, 4, (h // 8 + 1, w // 8 + 1)).repeat(8, 0).repeat(8, 1)[:h, :w]).astype(np.uint32)
    material = (part * 3 % 5).astype(np.uint32)
    depth = (np.float32(100.0) + rng.random((h, w), dtype=np.float32) * np.float32(5.0)).astype(np.float32)
    depth[part == 0] = np.inf
    depth[rng.random((h, w)) < 0.01] = np.nan
    normal = rng.normal(size=(h, w, 3)).astype(np.float32)
    normal /= np.linalg.norm(normal, axis=-1, keepdims=True).astype(np.float32)
    normal[rng.random((h, w)) < 0.01] = np.nan
    albedo = rng.random((h, w, 3), dtype=np.float32)
    albedo[rng.random((h, w)) < 0.05] = 0.0
    mean = rng.random((h, w, 3), dtype=np.float32) * np.float32(0.5)
    spikes = rng.random((h, w)) < 0.03
    mean[spikes] *= np.float32(200.0)
    mean[20, 30:34] = np.float32(500.0)  # a row of fireflies: each clamp reads the previous one's
    mean[21, 31] = np.float32(800.0)
    sums = np.concatenate([mean * np.float32(samples), np.ones((h, w, 1), np.float32) * np.float32(samples)], axis=-1).astype(np.float32)
    lum = (np.float32(0.2126) * mean[..., 0] + np.float32(0.7152) * mean[..., 1]).astype(np.float32) + np.float32(0.0722) * mean[..., 2]
    lum2 = ((lum * lum + rng.random((h, w), dtype=np.float32)) * np.float32(samples)).astype(np.float32)
    words = oracle_lib.denoise_words(sums, lum2, albedo, normal, depth, part, material)
    for preset in (0, 1):
        a = rtg.denoise(words, w, h, samples, preset=preset)
        b = oracle_lib.denoise(words, w, h, samples, preset=preset)
        assert np.array_equal(bits(a), bits(b)), preset
    assert n == w * h


@pytest.mark.parametrize("name, capacity", [("example", 0), ("e11 small", 0), ("e11 small", 5000)])
def test_fused_guides_are_the_traced_ones(rtg, pins, name, capacity):
    """rtg_film_guides_fused: the albedo read from the render's own first hits (edge pixels the
    mean of their sub-samples, in waves of any size) gives rtg_film_guides' guides bit for bit,
    so the same denoised image, and leaves the film itself as it was."""
    from repackshot_b200 import scenes
    sc = scenes.example_scene() if name == "example" else scenes.e11_scene()
    if name != "example":
        sc.width, sc.height = 160, 120
    s = rtg.Scene(scenes.to_rsb(sc))
    if capacity:
        s.set_path_capacity(capacity)
    a = s.film()
    a.render(0, 4)
    a.guides(0, 4)
    b = s.film()
    b.fuse_guides()
    b.render(0, 1)
    b.render(1, 3)
    for x, y in zip(a.read(), b.read()):
        assert np.array_equal(bits(x), bits(y))
    da, db = a.denoise(4), b.denoise(4)
    assert np.array_equal(bits(da), bits(db))
    if name == "example":
        assert fnv1a_floats(means(db, 4)) == pins["denoised"]["example_4spp"]


def test_an_adaptive_film_is_denoised_with_its_own_counts(rtg, oracle_lib):
    """An adaptive film (pixels with their own counts) denoised on the device equals the oracle's
    denoiser on its sums rescaled to `samples` samples with the counts plane (rt-cli/src/lib.rs:104,
    adaptive.rs:260), also at half strength."""
    from repackshot_b200 import scenes
    sc = scenes.example_scene()
    sc.width, sc.height = 96, 64
    sc.adaptive, sc.noise_threshold = 1, 0.05
    rsb = scenes.to_rsb(sc)
    s = rtg.Scene(rsb)
    f = s.film()
    ad = rtg.Adaptive(s, f, 48)
    ad.run(0)
    ad.close()
    samples = 48
    f.guides(0, 16)
    rgb, weight, alpha, lum2 = f.read()
    assert weight.min() < weight.max()
    f32 = np.float32

    def rescale(x):
        x = np.asarray(x, f32)
        wt = weight if x.ndim == 2 else weight[..., None]
        scaled = ((x * (f32(1.0) / np.where(wt > 0, wt, f32(1.0)))).astype(f32) * f32(samples)).astype(f32)
        return np.where(wt == f32(samples), x, np.where(wt > 0, scaled, f32(0.0))).astype(f32)

    sums = np.concatenate([rescale(rgb), rescale(alpha)[..., None]], axis=-1)
    albedo, normal, depth, part, material = oracle_lib.OracleScene(rsb).guides(16)
    words = oracle_lib.denoise_words(sums, rescale(lum2), albedo, normal, depth, part, material, counts=weight)
    for strength in (1.0, 0.5):
        want = oracle_lib.denoise(words, 96, 64, samples, strength=strength)
        got = f.denoise(samples, strength=strength)
        assert np.array_equal(bits(got).reshape(-1), bits(want))
