"""The oracle's IES profiles and IES lights against the reference's known answers: the unit tests of
engine/crates/rt-core/src/ies/tests.rs (the two hand-written files, nodes and bilinear values, the
horizontal angle's direction, the flux of an isotropic and of a cos^2 lamp, refusals), restated
with the same inputs and tolerances; and the L5 scene (the example lit by a downlight sphere and a
wall-washer point), whose file is the reference's fixture byte for byte and whose 4-sample film has
the reference's pinned hash (render.rs:1510-1531). The two profiles are the reference's test files,
kept in tests/golden/ies_profiles.json by tests/golden/make_golden.py.
"""
import hashlib
import json
import math
from pathlib import Path

import numpy as np
import pytest

from repackshot_b200 import scenes

PROFILES = json.loads((Path(__file__).resolve().parent / "golden" / "ies_profiles.json").read_text())
DOWNLIGHT, WALL_WASHER = PROFILES["downlight-symmetric"], PROFILES["wall-washer"]


def fmt(x):
    """A float as Rust's `{}` prints an f32 (the shortest text that reads back to it)."""
    x = float(np.float32(x))
    if x == int(x) and abs(x) < 1e16:
        return str(int(x))
    return repr(float(np.float32(x))).rstrip("0") if "e" not in repr(x) else repr(x)


def ies_text(vertical, horizontal, f):
    """ies/tests.rs:14: a type C file with these angles and candela f(gamma, phi)."""
    join = lambda v: " ".join(fmt(x) for x in v)
    text = "IESNA:LM-63-2002\n[LUMINAIRE] generated\nTILT=NONE\n"
    text += f"1 1000 1 {len(vertical)} {len(horizontal)} 1 2 0 0 0\n1 1 10\n{join(vertical)}\n{join(horizontal)}\n"
    for h in horizontal:
        text += join([f(v, h) for v in vertical]) + "\n"
    return text


def angles(a, b, step):
    n = round((b - a) / step)
    return [a + step * i for i in range(n + 1)]


def direction(gamma, phi):
    g, p = math.radians(gamma), math.radians(phi)
    return (math.sin(g) * math.sin(p), math.sin(g) * math.cos(p), math.cos(g))


def test_downlight_nodes_and_interpolation(oracle_lib):
    pts = [(g, phi) for g in (0.0, 30.0, 60.0, 90.0) for phi in (0.0, 123.0)] + [(35.0, 0.0)]
    dirs = [direction(g, 77.0) for g in (0.0, 30.0, 60.0, 90.0)]
    peak, flux, sym, inten, shape = oracle_lib.ies(DOWNLIGHT, pts, dirs)
    assert peak == 1000.0 and sym == 0
    want = [1000.0, 1000.0, 750.0, 750.0, 250.0, 250.0, 0.0, 0.0, 668.5]
    assert np.all(np.abs(inten - np.array(want, np.float32)) <= 1.0e-3)
    assert np.all(np.abs(shape * 1000.0 - np.array([1000.0, 750.0, 250.0, 0.0], np.float32)) <= 0.1)
    _, _, _, outside, _ = oracle_lib.ies(DOWNLIGHT, [(90.001, 0.0), (95.0, 0.0), (180.0, 0.0), (-1.0, 0.0), (float("nan"), 0.0)])
    assert np.all(outside == 0.0)
    exact = 2.0 * math.pi * 1000.0 / 3.0
    assert abs(flux / exact - 1.0) <= 6.0e-3


def test_wall_washer_follows_its_table(oracle_lib):
    pts = [(60.0, 0.0), (60.0, 90.0), (60.0, 180.0), (60.0, 270.0), (60.0, 360.0), (30.0, 0.0), (30.0, 45.0), (30.0, 405.0),
           (30.0, -45.0)]
    plus_x = (math.sin(math.radians(60.0)), 0.0, math.cos(math.radians(60.0)))
    peak, _, sym, inten, shape = oracle_lib.ies(WALL_WASHER, pts, [plus_x, (0.0, 0.0, 1.0)])
    assert peak == 900.0 and sym == 4
    want = [560.0, 430.0, 330.0, 380.0, 560.0, 800.0, 765.0, 765.0, 0.5 * (800.0 + 0.5 * (800.0 + 600.0))]
    assert np.all(np.abs(inten - np.array(want, np.float32)) <= 1.0e-3)
    assert abs(shape[0] - 430.0 / 900.0) <= 1.0e-6 and shape[1] == 1.0
    # the horizontal angle runs from +y towards +x
    _, _, _, _, sides = oracle_lib.ies(WALL_WASHER, (), [direction(60.0, p) for p in (0.0, 90.0, 180.0, 270.0)])
    assert np.all(np.abs(sides * 900.0 - np.array([560.0, 430.0, 330.0, 380.0], np.float32)) <= 0.05)


def test_flux_of_isotropic_and_cosine_squared_lamps(oracle_lib):
    exact = 4.0 * math.pi * 100.0
    _, flux, _, _, _ = oracle_lib.ies(ies_text(angles(0.0, 180.0, 10.0), [0.0], lambda g, p: 100.0))
    assert abs(flux - exact) <= exact * 2.0e-6
    v = [0.0, 3.0, 17.0, 40.0, 41.0, 90.0, 120.0, 179.0, 180.0]
    for h in ([0.0], [0.0, 20.0, 90.0], [0.0, 70.0, 180.0], [90.0, 200.0, 270.0], [0.0, 100.0, 250.0, 360.0]):
        _, flux, _, _, _ = oracle_lib.ies(ies_text(v, h, lambda g, p: 100.0))
        assert abs(flux - exact) <= exact * 4.0e-6, h
    _, half, _, _, _ = oracle_lib.ies(ies_text(angles(0.0, 90.0, 15.0), [0.0], lambda g, p: 100.0))
    assert abs(half - 2.0 * math.pi * 100.0) <= 1.0e-3
    fine = ies_text(angles(0.0, 90.0, 1.0), [0.0], lambda g, p: np.float32(1000.0 * math.cos(math.radians(g)) ** 2))
    _, flux, _, _, _ = oracle_lib.ies(fine)
    assert abs(flux / (2.0 * math.pi * 1000.0 / 3.0) - 1.0) <= 1.0e-4


@pytest.mark.parametrize("edit, words", [
    (lambda t: t.replace("TILT=NONE", "TILT=INCLUDE"), "TILT=INCLUDE"),
    (lambda t: t.replace("TILT=NONE", "TILT=lamp.tlt"), "TILT file"),
    (lambda t: t.replace("TILT=NONE\n", ""), "no TILT"),
    (lambda t: t.replace("1 2094 1 10 1 1 2 0 0 0", "1 2094 1 10 1 2 2 0 0 0"), "type C"),
    (lambda t: t.replace("1 2094 1 10 1 1 2 0 0 0", "1 2094 1 11 1 1 2 0 0 0"), "fewer values"),
    (lambda t: t.replace("1000 970", "-1000 970"), "negative"),
    (lambda t: t.replace("1000 970", "x 970"), "not a number"),
    (lambda t: t.replace("1 2094 1 10 1 1 2 0 0 0", "1 2094 0 10 1 1 2 0 0 0"), "multiplier"),
])
def test_bad_files_are_refused_with_the_reason(oracle_lib, edit, words):
    bad = edit(DOWNLIGHT)
    assert bad != DOWNLIGHT
    with pytest.raises(ValueError, match=words):
        oracle_lib.ies(bad)


@pytest.fixture(scope="module")
def l5_rsb():
    return scenes.to_rsb(scenes.l5_scene(DOWNLIGHT.encode(), WALL_WASHER.encode()))


def test_l5_scene_bytes_are_the_reference_fixture(l5_rsb, pins):
    assert len(l5_rsb) == pins["l5_rsb"]["bytes"]
    assert hashlib.sha256(l5_rsb).hexdigest() == pins["l5_rsb"]["sha256"]


def test_l5_at_four_samples_has_the_pinned_hash(oracle_lib, l5_rsb, pins):
    o = oracle_lib.OracleScene(l5_rsb)
    rgb, w, _, _, _ = o.render_film(0, 4, threads=8)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["l5_ies_4spp"]


def test_ies_light_without_profile_is_refused(oracle_lib):
    s = scenes.l5_scene(DOWNLIGHT.encode(), WALL_WASHER.encode())
    s.lights[2].profile = 7
    with pytest.raises(ValueError, match="IESP"):
        oracle_lib.OracleScene(scenes.to_rsb(s))
