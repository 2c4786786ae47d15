"""The oracle's denoiser (engine/crates/rt-post/src/denoise.rs) against the reference's known
answers: the denoised example's pinned hashes (the full filter at 4 samples, the viewport's at 2
and 4: denoise/tests.rs:369-528), bands of rows giving those rows of the whole image
(tests.rs:184), strength 0 and 0.5 (tests.rs:533), the halos, and refusals (tests.rs:210)."""
import numpy as np
import pytest

from denoise_cases import example_input, fnv1a_floats, means


@pytest.fixture(scope="module")
def example4(oracle_lib):
    return example_input(oracle_lib, 4)


def test_the_denoised_example_has_the_pinned_hash(oracle_lib, example4, pins):
    o, words, (rgb, alpha, lum2), _ = example4
    out = oracle_lib.denoise(words, o.width, o.height, 4)
    assert fnv1a_floats(means(out, 4)) == pins["denoised"]["example_4spp"]
    # without denoise the image keeps its own pin
    inv = np.float32(1.0) / np.float32(4)
    assert fnv1a_floats((rgb * inv).astype(np.float32)) == pins["film_hashes"]["example_4spp"]


def test_the_viewport_preset_has_the_pinned_hashes(oracle_lib, example4, pins):
    o, words, _, _ = example4
    assert fnv1a_floats(means(oracle_lib.denoise(words, o.width, o.height, 4, preset=1), 4)) == pins["denoised"]["viewport_example_4spp"]
    o2, words2, _, _ = example_input(oracle_lib, 2)
    assert fnv1a_floats(means(oracle_lib.denoise(words2, o2.width, o2.height, 2, preset=1), 2)) == pins["denoised"]["viewport_example_2spp"]


def band_words(words, width, height, lo, hi):
    """The planes of rows lo..hi of whole-image input words (14 a pixel)."""
    n = width * height
    out = []
    for start, ch in ((0, 4), (4 * n, 1), (5 * n, 3), (8 * n, 3), (11 * n, 1), (12 * n, 1), (13 * n, 1)):
        plane = words[start:start + n * ch].reshape(height, width * ch)
        out.append(plane[lo:hi].reshape(-1))
    return np.concatenate(out)


def test_a_band_of_rows_is_exactly_those_rows(oracle_lib, example4):
    o, words, _, _ = example4
    w, h = o.width, o.height
    whole = oracle_lib.denoise(words, w, h, 4)
    halo = oracle_lib.denoise_halo(0)
    assert halo == 72 and oracle_lib.denoise_halo(1) == 24 and oracle_lib.denoise_halo(2) == 0
    parts = []
    for k in range(5):
        y0, y1 = h * k // 5, h * (k + 1) // 5
        lo, hi = max(0, y0 - halo), min(h, y1 + halo)
        parts.append(oracle_lib.denoise(band_words(words, w, h, lo, hi), w, h, 4, origin_y=lo, rows=hi - lo, y0=y0, y1=y1))
    assert np.array_equal(np.concatenate(parts).view(np.uint32), whole.view(np.uint32))
    with pytest.raises(ValueError, match="status 5"):  # a band without its halo
        oracle_lib.denoise(band_words(words, w, h, 100, 200), w, h, 4, origin_y=100, rows=100, y0=120, y1=180)
    with pytest.raises(ValueError, match="status 5"):
        oracle_lib.denoise(words, w, h, 4, preset=7)


def test_strength(oracle_lib, example4):
    o, words, _, _ = example4
    n = o.width * o.height
    noisy = words[:4 * n].view(np.float32)
    full = oracle_lib.denoise(words, o.width, o.height, 4)
    assert np.array_equal(oracle_lib.denoise(words, o.width, o.height, 4, strength=0.0).view(np.uint32), noisy.view(np.uint32))
    assert np.array_equal(oracle_lib.denoise(words, o.width, o.height, 4, strength=float("nan")).view(np.uint32), full.view(np.uint32))
    half = oracle_lib.denoise(words, o.width, o.height, 4, strength=0.5).reshape(-1, 4)
    want = (noisy.reshape(-1, 4) * np.float32(0.5) + full.reshape(-1, 4) * np.float32(0.5)).astype(np.float32)
    assert np.array_equal(half[:, :3], want[:, :3]) and np.array_equal(half[:, 3], noisy.reshape(-1, 4)[:, 3])
