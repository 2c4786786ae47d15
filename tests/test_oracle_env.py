"""The oracle's bitmaps, Radiance files, 2-D distribution and HDRI scene against the reference's
own known answers: the unit tests of engine/crates/rt-core/src/bitmap.rs
(raw_formats_decode_and_check_their_size, encoded_files_decode_and_wide_images_are_halved,
bilinear_lookups_hit_pixel_centres_and_wrap, the_2d_distribution_samples_in_proportion_and_knows_its_density)
and hdr.rs (rgbe_pixels_round_trip_exactly, files_round_trip_through_the_writer,
flat_and_old_rle_scanlines_and_bottom_up_files_read, bad_files_fail_cleanly), restated with the
same inputs and tolerances; and the E5 scene (clear glass, coat, anisotropy, a thin glass card, a
cut-out card, an HDRI over a background image), whose file is the reference's fixture byte for
byte and whose 4-sample film has the reference's pinned FNV-1a hash (render.rs:1086-1107), and
the same scene under the classic sky with a sun, also pinned.
"""
import hashlib
from pathlib import Path
import struct

import numpy as np
import pytest

from repackshot_b200 import scenes


def test_raw_formats_decode_and_check_their_size(oracle_lib):
    tex, _ = oracle_lib.bitmap(0, 2, 1, bytes([0, 128, 255, 255, 0, 0]))
    assert tex[0, 0, 0] == 0.0 and abs(tex[0, 0, 1] - 0.215861) < 1.0e-5 and tex[0, 0, 2] == 1.0
    assert list(tex[0, 1]) == [1.0, 0.0, 0.0]
    tex, _ = oracle_lib.bitmap(1, 1, 1, bytes([255, 0, 0, 7]))
    assert list(tex[0, 0]) == [1.0, 0.0, 0.0]
    tex, _ = oracle_lib.bitmap(2, 1, 2, struct.pack("<6f", 1.0, 2.0, 3.0, -1.0, float("nan"), 5.0))
    assert list(tex[0, 0]) == [1.0, 2.0, 3.0] and list(tex[1, 0]) == [0.0, 0.0, 5.0]
    for fmt, w, h, data, why in [(0, 2, 2, bytes(6), "size"), (0, 0, 0, b"", "size"), (99, 1, 1, bytes(3), "unknown")]:
        with pytest.raises(ValueError, match=why):
            oracle_lib.bitmap(fmt, w, h, data)


def test_encoded_files_decode_and_wide_images_are_halved(oracle_lib):
    w, h = 4096 + 2, 3
    rgb = (np.arange(3 * w * h) % 5).astype(np.float32)
    f = scenes.hdr_encode(w, h, rgb)
    tex, _ = oracle_lib.bitmap(16, 0, 0, f)
    assert tex.shape[:2] == (2, (w + 1) // 2)
    with pytest.raises(ValueError, match="size"):
        oracle_lib.bitmap(16, 5, 5, f)


def test_bilinear_lookups_hit_pixel_centres_and_wrap(oracle_lib):
    data = struct.pack("<6f", 0.0, 0.0, 0.0, 1.0, 1.0, 1.0)
    _, out = oracle_lib.bitmap(2, 2, 1, data, [(0.25, 0.5, 0), (0.75, 0.5, 0), (0.5, 0.5, 0), (1.0, 0.5, 0), (1.0, 0.5, 1),
                                               (0.0, 0.5, 1)])
    assert list(out[:, 0]) == [0.0, 1.0, 0.5, 1.0, 0.5, 0.5]


def test_2d_distribution_samples_in_proportion_and_knows_its_density(oracle_lib):
    w, h = 8, 4
    weights = np.array([(i * 7) % 5 for i in range(w * h)], np.float32)
    rng = np.random.default_rng(5)
    n = 400_000
    out = oracle_lib.dist2d(w, h, weights, rng.random((n, 2), dtype=np.float32))
    u, v, pdf, pdf_at = out.T
    assert np.all((u >= 0) & (u < 1) & (v >= 0) & (v < 1))
    assert np.all(np.abs(pdf - pdf_at) < 1.0e-5 * np.maximum(pdf, 1.0))
    cells = (v * h).astype(int) * w + (u * w).astype(int)
    counts = np.bincount(cells, minlength=w * h)
    want = weights / weights.sum()
    assert np.all(np.abs(counts / n - want) < 0.003)
    assert np.all(counts[weights == 0] == 0)
    assert oracle_lib.dist2d(2, 2, np.zeros(4, np.float32), [(0.5, 0.5)]) is None


def _rgbe_to_rgb(p):
    if p[3] == 0:
        return np.zeros(3, np.float32)
    f = np.float32(2.0) ** np.float32(int(p[3]) - 136)
    return np.array([p[0], p[1], p[2]], np.float32) * f


def test_rgbe_and_files_round_trip(oracle_lib):
    assert scenes._rgb_to_rgbe([1.0, 0.5, 0.25]) == bytes([128, 64, 32, 129])
    assert scenes._rgb_to_rgbe([0.0, -1.0, float("nan")]) == bytes(4)
    rng = np.random.default_rng(7)
    for w, h in [(1, 1), (7, 3), (8, 2), (64, 32), (300, 5)]:
        rgb = (rng.random((h, w, 3), dtype=np.float32) * np.float32(4.0)).astype(np.float32)
        f = scenes.hdr_encode(w, h, rgb)
        assert f.startswith(b"#?RADIANCE\n")
        tex, _ = oracle_lib.bitmap(16, 0, 0, f)
        want = np.array([[_rgbe_to_rgb(scenes._rgb_to_rgbe(rgb[y, x])) for x in range(w)] for y in range(h)], np.float32)
        assert np.array_equal(tex, want)
        assert scenes.hdr_encode(w, h, tex) == f
        if w >= 64:
            assert len(scenes.hdr_encode(w, h, np.full((h, w, 3), 0.5, np.float32))) < 4 * w * h


def test_flat_and_old_rle_scanlines_and_bottom_up_files_read(oracle_lib):
    f = b"#?RGBE\nGAMMA=1\nEXPOSURE=2\n\n+Y 2 +X 3\n"
    f += bytes([128, 128, 128, 129, 1, 1, 1, 2])
    f += bytes([128, 0, 0, 129, 0, 128, 0, 129, 0, 0, 128, 129])
    tex, _ = oracle_lib.bitmap(16, 0, 0, f)
    assert list(tex[0].reshape(-1)) == [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    assert list(tex[1].reshape(-1)) == [1.0] * 9


def test_bad_files_fail_cleanly(oracle_lib):
    for f in [b"P6\n", b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n\n-Y 1 +X 1\n\0\0\0\0", b"#?RADIANCE\n\n-X 1 +Y 1\n\0\0\0\0"]:
        with pytest.raises(ValueError):
            oracle_lib.bitmap(16, 0, 0, f)
    rng = np.random.default_rng(3)
    f = scenes.hdr_encode(64, 4, rng.random((4, 64, 3), dtype=np.float32))
    for cut in range(len(f)):
        with pytest.raises(ValueError):
            oracle_lib.bitmap(16, 0, 0, f[:cut])
    start = f.index(bytes([2, 2, 0, 64]))
    bad = bytearray(f)
    bad[start + 4] = 255
    with pytest.raises(ValueError):
        oracle_lib.bitmap(16, 0, 0, bytes(bad))


def test_exr_bitmaps_are_refused(oracle_lib):
    with pytest.raises(ValueError, match="unsupported: OpenEXR"):
        oracle_lib.bitmap(17, 0, 0, b"v/1\x01")


@pytest.fixture(scope="module")
def e5_rsb():
    return scenes.to_rsb(scenes.e5_scene())


def test_e5_scene_bytes_are_the_reference_fixture(e5_rsb, pins):
    assert len(e5_rsb) == pins["e5_rsb"]["bytes"]
    assert hashlib.sha256(e5_rsb).hexdigest() == pins["e5_rsb"]["sha256"]


def test_e5_at_four_samples_has_the_pinned_hash(oracle_lib, e5_rsb, pins):
    s = oracle_lib.OracleScene(e5_rsb)
    rgb, w, _, _, _ = s.render_film(0, 4, tile=32, threads=4)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["e5_hdri_4spp"]


def test_e5_under_the_classic_sky_has_the_pinned_hash(oracle_lib, pins):
    s = oracle_lib.OracleScene(scenes.to_rsb(scenes.e5_scene(sky=True)))
    rgb, w, _, _, _ = s.render_film(0, 4, tile=32, threads=4)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["e5_sky_4spp"]


def test_e5c_under_the_physical_sky_has_the_pinned_hash(oracle_lib, pins):
    # render.rs:1112-1128: the physical sky (the fitted Hosek-Wilkie table) at 4 spp.
    s = oracle_lib.OracleScene(scenes.to_rsb(scenes.e5c_scene()))
    rgb, w, _, _, _ = s.render_film(0, 4, tile=32, threads=4)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["e5c_physical_sky_4spp"]


def test_the_physical_sky_table_is_the_published_one():
    # The table the product compiles in and the oracle loads: SHA-256 as sky_table.rs states it.
    data = (Path(__file__).resolve().parent.parent / "repackshot_b200" / "data" / "sky_table.f32").read_bytes()
    assert len(data) == 4 * 3600
    assert hashlib.sha256(data).hexdigest() == "2329ac7376204749a317d5b31e23e17fa27950515be0f0d50018cd9c16e8a721"


def test_bad_bitmap_indices_are_refused(oracle_lib):
    s = scenes.e5_scene()
    s.hdri_map = 2
    with pytest.raises(ValueError, match="bitmap index"):
        oracle_lib.OracleScene(scenes.to_rsb(s))
