"""The oracle's adaptive sampling (E10) against the reference's known answers, restated from
engine/crates/rt-core/src/adaptive/tests.rs with the same inputs and bounds: the relative error of a
pixel, the blocks a decision chooses and the size of the round, the pinned hash of six decisions
over the synthetic image (tests.rs:534), and the property that every pixel of an adaptive image is
bit for bit the plain mean of its own samples (tests.rs:391, the example at 48 x 40 with a 3 %
target and a cap of 96)."""
import math

import numpy as np
import pytest

from adaptive_cases import grey, half_noisy, one_noisy_block, synthetic_decisions, words_as_floats
from repackshot_b200 import scenes

EPS = 0.01


def test_the_error_of_a_pixel_is_the_relative_error_of_its_mean(oracle_lib):
    pe = oracle_lib.pixel_error
    s, l2 = grey(16, 0.5, 0.0)
    assert pe(s, s, s, l2, 16, EPS) == 0.0
    s, l2 = grey(16, 0.5, 0.1)
    e = pe(s, s, s, l2, 16, EPS)
    want = math.sqrt(np.float32(0.01) / np.float32(15.0)) / 0.51
    assert abs(e - want) < 1.0e-4 * want
    s64, l64 = grey(64, 0.5, 0.1)
    assert abs(pe(s64, s64, s64, l64, 64, EPS) / e - 0.5) < 0.02
    assert pe(1.0, 1.0, 1.0, 1.0, 1, EPS) == np.float32(1.0e30)
    assert pe(float("nan"), 1.0, 1.0, 1.0, 8, EPS) == np.float32(1.0e30)
    assert pe(1.0, 1.0, 1.0, float("inf"), 8, EPS) == np.float32(1.0e30)


def test_the_next_round_goes_to_the_noisy_blocks_above_the_median(oracle_lib):
    w, h = 64, 16
    counts = np.full(16, 16, np.uint32)
    sums, lum2 = half_noisy(w, h, 32, 0.2, 16)
    active, words = oracle_lib.adaptive_decide(w, h, 0.0, 0.0, 0, counts, sums, lum2)
    threshold, max_error, _ = words_as_floats(words)
    assert words[2] == 16 and threshold > 0.0 and max_error >= threshold
    assert all(b % 8 < 4 for b in range(16) if active[b])
    assert words[1] >= 4 and words[0] == 16
    active, words = oracle_lib.adaptive_decide(w, h, 0.0, 0.5, 0, counts, sums, lum2)
    assert (words[0], words[1]) == (0, 0) and not active.any() and words_as_floats(words)[2] == 0.0
    clean, clean2 = half_noisy(w, h, 0, 0.0, 16)
    _, words = oracle_lib.adaptive_decide(w, h, 0.0, 0.0, 0, counts, clean, clean2)
    assert words[0] == 0 and words_as_floats(words)[1] == 0.0
    _, words = oracle_lib.adaptive_decide(w, h, 0.0, 0.0, 16, counts, sums, lum2)
    assert words[0] == 0


def test_a_noisier_block_wins_and_few_active_blocks_take_longer_rounds(oracle_lib):
    counts = np.full(64, 16, np.uint32)
    sums, lum2 = one_noisy_block(counts)
    active, words = oracle_lib.adaptive_decide(64, 64, 0.0, 0.06, 0, counts, sums, lum2)
    assert words[1] == 1 and active[0] and words[0] == 16
    counts[0] = 400
    s400, l400 = one_noisy_block(counts)
    active, words = oracle_lib.adaptive_decide(64, 64, 0.0, 0.02, 0, counts, s400, l400)
    assert words[1] == 1 and active[0] and words[0] == 16 * 16
    counts[0] = 16
    _, words = oracle_lib.adaptive_decide(64, 64, 0.0, 0.01, 0, counts, sums, lum2)
    assert words_as_floats(words)[2] > 64.0 * 16.0 * 200.0
    _, words = oracle_lib.adaptive_decide(64, 64, 0.0, 0.01, 100, counts, sums, lum2)
    assert 0.0 < words_as_floats(words)[2] <= 4.0 * 84.0 * 64.0


def test_bad_planes_are_refused(oracle_lib):
    with pytest.raises(ValueError, match="status 2"):
        oracle_lib.adaptive_decide(0, 0, 0.0, 0.0, 0, np.zeros(0), np.zeros(0), np.zeros(0))


def test_the_decisions_of_a_synthetic_image_have_the_pinned_hash(oracle_lib, pins):
    assert synthetic_decisions(oracle_lib.adaptive_decide, 6) == pins["e10_synthetic_decisions"]


def adaptive_example():
    s = scenes.example_scene()
    s.width, s.height = 48, 40
    s.adaptive, s.noise_threshold = 1, 0.03
    return s


def test_adaptive_render_section_is_the_reference_layout():
    plain = scenes.to_rsb(scenes.example_scene())
    rsb = scenes.to_rsb(adaptive_example())
    assert len(rsb) == len(plain) + 8  # RNDR grows from 64 to 72 bytes (rsb.rs:1968)


def test_every_pixel_of_an_adaptive_image_is_the_plain_mean_of_its_own_samples(oracle_lib):
    o = oracle_lib.OracleScene(scenes.to_rsb(adaptive_example()))
    rgb, weight, _, lum2, counts, (lo, hi, decisions, _) = o.adaptive_film(96, 16, threads=8)
    assert hi > lo and lo >= 16 and decisions >= 2
    per_pixel = np.repeat(np.repeat(counts, 8, axis=0), 8, axis=1)[:40, :48]
    assert np.array_equal(weight, per_pixel.astype(np.float32))
    checked = 0
    for n in np.unique(per_pixel):
        prgb, _, _, pl2, _ = o.render_film(0, int(n), threads=8)
        at = per_pixel == n
        assert np.array_equal(rgb[at].view(np.uint32), prgb[at].view(np.uint32)), n
        assert np.array_equal(lum2[at].view(np.uint32), pl2[at].view(np.uint32)), n
        checked += int(at.sum())
    assert checked == 48 * 40
