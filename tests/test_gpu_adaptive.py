"""Adaptive sampling (E10) on the GPU, through the C ABI, against the oracle and the reference's
known answers (engine/crates/rt-core/src/adaptive.rs and adaptive/tests.rs):

* rtg_adaptive_decide (block errors on the GPU, the per-block choice on the host) gives the oracle's
  bytes and words on the reference's test images and on random planes with unmeasurable pixels, and
  the reference's pinned hash of six decisions over the synthetic image (tests.rs:534);
* an adaptive render (rtg_adaptive_*) of the example at 48 x 40 with a 3 % target and a cap of 96 is
  bit for bit the oracle's adaptive film, for passes of 16, 5 and 3 samples and runs cut into single
  passes, and every pixel is the plain mean of its own samples (tests.rs:391);
* with edge samples and the Blackman-Harris filter (the E11 scene, small) likewise, and under a cap
  below the warm-up the image is the plain film of `cap` samples;
* rtg_render_block_rgba gives the pixels of rtg_render_tile_rgba and of the oracle.
"""
import numpy as np
import pytest

from adaptive_cases import half_noisy, one_noisy_block, synthetic_decisions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def same_decision(rtg, oracle_lib, *args):
    a1, w1 = rtg.adaptive_decide(*args)
    a2, w2 = oracle_lib.adaptive_decide(*args)
    assert np.array_equal(a1, a2) and np.array_equal(w1, w2), (w1, w2)
    return w1


def test_decisions_of_the_reference_images_are_the_oracle_ones(rtg, oracle_lib):
    counts = np.full(16, 16, np.uint32)
    sums, lum2 = half_noisy(64, 16, 32, 0.2, 16)
    for target, cap in ((0.0, 0), (0.5, 0), (0.0, 16), (0.01, 40)):
        same_decision(rtg, oracle_lib, 64, 16, 0.0, target, cap, counts, sums, lum2)
    counts = np.full(64, 16, np.uint32)
    counts[0] = 400
    sums, lum2 = one_noisy_block(counts)
    for target, cap in ((0.06, 0), (0.02, 0), (0.01, 0), (0.01, 100), (0.01, 500)):
        same_decision(rtg, oracle_lib, 64, 64, 0.0, target, cap, counts, sums, lum2)


@pytest.mark.parametrize("w, h, seed", [(45, 37, 1), (101, 67, 2), (8, 8, 3), (1, 129, 4), (333, 7, 5)])
def test_decisions_of_random_planes_are_the_oracle_ones(rtg, oracle_lib, w, h, seed):
    rng = np.random.default_rng(seed)
    cols, rows = (w + 7) // 8, (h + 7) // 8
    counts = rng.integers(0, 70, cols * rows).astype(np.uint32)
    n = np.repeat(np.repeat(counts.reshape(rows, cols), 8, 0), 8, 1)[:h, :w].astype(np.float32)
    mean = rng.random((h, w, 3), dtype=np.float32) * np.float32(rng.choice([0.01, 1.0, 50.0]))
    sums = np.concatenate([mean * n[..., None], n[..., None]], axis=-1).astype(np.float32)
    lum = (np.float32(0.2126) * mean[..., 0] + np.float32(0.7152) * mean[..., 1]).astype(np.float32) + np.float32(0.0722) * mean[..., 2]
    lum2 = ((lum * lum + rng.random((h, w), dtype=np.float32) * np.float32(0.3)) * n).astype(np.float32)
    bad = rng.random((h, w)) < 0.01
    sums[bad, 0] = np.float32("nan")
    lum2[rng.random((h, w)) < 0.01] = np.float32("inf")
    for ev, target, cap in ((0.0, 0.0, 0), (0.5, 0.02, 200), (-3.0, 0.1, 64), (12.0, 1.0, 0)):
        same_decision(rtg, oracle_lib, w, h, ev, target, cap, counts, sums, lum2)


def test_the_decisions_of_a_synthetic_image_have_the_pinned_hash(rtg, pins):
    assert synthetic_decisions(rtg.adaptive_decide, 6) == pins["e10_synthetic_decisions"]


def small_adaptive(edges=False):
    from repackshot_b200 import scenes
    s = scenes.e11_scene() if edges else scenes.example_scene()
    s.width, s.height = (64, 48) if edges else (48, 40)
    s.adaptive, s.noise_threshold = 1, (0.05 if edges else 0.03)
    return s


def gpu_adaptive(rtg, rsb, cap, pass_samples, single_passes=False, capacity=0):
    s = rtg.Scene(rsb)
    if capacity:
        s.set_path_capacity(capacity)
    f = s.film()
    ad = rtg.Adaptive(s, f, cap)
    if single_passes:
        while True:
            passes, _ = ad.run(pass_samples, 1)
            if passes == 0:
                break
    else:
        ad.run(pass_samples)
    st = ad.state()
    samples, _ = ad.counts()
    out = f.read()
    ad.close()
    return out, samples, st


@pytest.fixture(scope="module")
def example_oracle(oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(small_adaptive())
    return rsb, oracle_lib.OracleScene(rsb).adaptive_film(96, 16, threads=8)


def assert_same_film(gpu, oracle):
    for a, b in zip(gpu, oracle):
        assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("pass_samples, single, capacity", [(16, False, 0), (0, False, 0), (5, False, 0), (3, True, 0), (16, False, 700)])
def test_adaptive_film_is_the_oracle_film(rtg, example_oracle, pass_samples, single, capacity):
    rsb, (rgb, w, al, l2, counts, (lo, hi, decisions, _)) = example_oracle
    (grgb, gw, gal, gl2), samples, st = gpu_adaptive(rtg, rsb, 96, pass_samples, single, capacity)
    assert st["converged"] == 1 and (st["lo"], st["hi"], st["decisions"]) == (lo, hi, decisions)
    assert np.array_equal(samples, counts)
    assert_same_film((grgb, gw, gal, gl2), (rgb, w, al, l2))


def test_every_pixel_is_the_plain_mean_of_its_own_samples(rtg, example_oracle):
    rsb, (_, _, _, _, counts, (lo, hi, _, _)) = example_oracle
    (grgb, gw, _, gl2), _, _ = gpu_adaptive(rtg, rsb, 96, 16)
    per_pixel = np.repeat(np.repeat(counts, 8, 0), 8, 1)[:40, :48]
    assert hi > lo
    s = rtg.Scene(rsb)
    for n in np.unique(per_pixel):
        f = s.film()
        f.render(0, int(n))
        prgb, _, _, pl2 = f.read()
        at = per_pixel == n
        assert np.array_equal(grgb[at].view(np.uint32), prgb[at].view(np.uint32))
        assert np.array_equal(gl2[at].view(np.uint32), pl2[at].view(np.uint32))


def test_adaptive_with_edge_samples_is_the_oracle_film(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(small_adaptive(edges=True))
    rgb, w, al, l2, counts, (lo, hi, decisions, _) = oracle_lib.OracleScene(rsb).adaptive_film(48, 16, threads=8)
    assert hi > lo
    for pass_samples in (16, 7):
        film, samples, st = gpu_adaptive(rtg, rsb, 48, pass_samples)
        assert (st["lo"], st["hi"], st["decisions"]) == (lo, hi, decisions)
        assert np.array_equal(samples, counts)
        assert_same_film(film, (rgb, w, al, l2))


def test_a_cap_below_the_warm_up_is_the_plain_film(rtg):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(small_adaptive())
    film, samples, st = gpu_adaptive(rtg, rsb, 6, 4)
    assert st["converged"] == 1 and st["lo"] == st["hi"] == 6 and np.all(samples == 6)
    f = rtg.Scene(rsb).film()
    f.render(0, 6)
    assert_same_film(film, f.read())


def test_render_block_rgba_is_the_tile_render(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(small_adaptive(edges=True))
    s = rtg.Scene(rsb)
    o = oracle_lib.OracleScene(rsb)
    for x, y, w, h, index in ((8, 16, 8, 8, 21), (56, 40, 8, 8, 3), (0, 0, 13, 5, 0)):
        st, block = rtg.render_block_rgba(s.handle, x, y, w, h, index, 7)
        assert st == rtg.STATUS_OK
        st, tile = rtg.render_tile(s.handle, x, y, w, h, index, rgba=True)
        assert np.array_equal(block.view(np.uint32), tile.view(np.uint32))
        assert np.array_equal(block.view(np.uint32), o.render_tile(x, y, w, h, index, rgba=True).view(np.uint32))
