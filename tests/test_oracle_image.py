"""The oracle's film output (exposure, tone curves, sRGB encoding; oracle/orc_image.cpp) against
the known answers of the reference's own tests (engine/crates/rt-core/src/color.rs:275-400), and
the PNG writer on a round trip. No GPU."""
import numpy as np
import pytest


def test_exposure_is_a_power_of_two(oracle_lib):  # color.rs: exposure_is_a_power_of_two
    assert list(oracle_lib.color(0, [0.0, 1.0, -1.0, 3.0])) == [1.0, 2.0, 0.5, 8.0]


def test_aces_known_values(oracle_lib):  # aces_maps_zero_to_zero_and_one_to_the_known_value
    z, one, neg = oracle_lib.color(1, [0.0, 1.0, -3.0])
    assert z == 0.0 and neg == 0.0
    assert abs(one - 0.803797) < 1e-4
    xs = np.linspace(0.0, 50.0, 2001, dtype=np.float32)  # aces_is_monotonic_bounded_and_clamps_negatives
    ys = oracle_lib.color(1, xs)
    assert np.all((ys >= 0) & (ys <= 1)) and np.all(np.diff(ys) >= 0)


def test_srgb_encode_matches_the_standard(oracle_lib):  # srgb_encode_matches_the_standard
    v = oracle_lib.color(2, [0.0, 1.0, 0.5, 0.002, -1.0, 5.0])
    assert v[0] == 0.0 and abs(v[1] - 1.0) < 1e-6 and abs(v[2] - 0.735357) < 1e-4
    assert abs(v[3] - np.float32(0.002) * np.float32(12.92)) < 1e-7 and v[4] == 0.0 and abs(v[5] - 1.0) < 1e-6


@pytest.mark.parametrize("kind", [2, 3])  # filmic_and_agx_put_middle_grey_mid_scale_and_keep_greys_neutral
def test_filmic_and_agx_grey(oracle_lib, kind):
    grey, bright, brighter, black = oracle_lib.color(3 + kind, np.float32([0.18, 0.18 * 16, 0.18 * 128, 0.0]))
    encoded = oracle_lib.color(2, [grey])[0]
    assert 0.42 < encoded < 0.56
    assert bright < 0.97 and brighter > 0.9 and black == 0.0


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])  # tonemaps_are_bounded_and_monotonic (per grey)
def test_curves_are_bounded_and_monotonic(oracle_lib, kind):
    xs = np.float32(np.geomspace(1e-4, 1e3, 400))
    ys = oracle_lib.color(3 + kind, xs)
    if kind != 0:
        assert np.all((ys >= 0) & (ys <= 1))
    assert np.all(np.diff(ys) >= -1e-7)


def test_agx_outset_inverts_the_inset(oracle_lib):
    assert np.allclose(oracle_lib.agx_identity(), np.eye(3), atol=1e-5)


def test_encode_quantises_as_the_reference(oracle_lib):
    # One pixel of sums (2, 1, 0.5) over weight 2, no exposure, linear curve: (1, 0.5, 0.25)
    # encoded to sRGB and then v * 255 + 0.5 truncated; an empty pixel is black.
    b8, b16 = oracle_lib.film_encode(np.float32([2.0, 1.0, 0.5, 0, 0, 0]), np.float32([2.0, 0.0]), 0.0, 0)
    enc = oracle_lib.color(2, [1.0, 0.5, 0.25])
    assert list(b8[0]) == [int(e * np.float32(255) + np.float32(0.5)) for e in enc]
    assert list(b16[0]) == [int(e * np.float32(65535) + np.float32(0.5)) for e in enc]
    assert list(b8[1]) == [0, 0, 0] and list(b16[1]) == [0, 0, 0]


def test_linear_film_is_the_resolve_times_the_exposure(oracle_lib):
    # Film::to_linear_exposed (image.rs:218): rgb * (1 / weight) * 2^ev, black where no sample, no
    # clamp: a pixel of 3 over weight 2 at +2 stops is 6.
    rgb = np.float32([2.0, 1.0, 0.5, 0, 0, 0, 3.0, 0.25, 7.0])
    wt = np.float32([2.0, 0.0, 2.0])
    for ev in (0.0, 2.0, -3.0):
        want = (rgb.reshape(3, 3) * np.float32([0.5, 0.0, 0.5])[:, None] * np.float32(2.0 ** ev)).astype(np.float32)
        assert np.array_equal(oracle_lib.film_linear(rgb, wt, ev), want)


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_png_round_trip(dtype):
    from repackshot_b200.image import png_bytes, read_png
    rng = np.random.default_rng(4)
    img = rng.integers(0, np.iinfo(dtype).max, (7, 13, 3), endpoint=True).astype(dtype)
    data = png_bytes(img)
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    back = read_png(data)
    assert back.dtype == dtype and np.array_equal(back, img)
