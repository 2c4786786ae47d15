"""The oracle against the reference's own known answers (tests/golden/reference_pins.json, read
from the reference tree by tests/golden/make_golden.py): the pinned film hashes of the example
scene, the PCG32 and mix64 values, the first Sobol points, the six energy tables, and the exact
passes with the 4-sample albedo and alpha of the example and the E5 example."""
import hashlib
import struct

import numpy as np
import pytest


def test_pcg32_and_mix64(oracle_lib, pins):
    out = np.zeros(6, np.uint32)
    oracle_lib.lib().orc_pcg32(42, 54, 6, oracle_lib._p(out))
    assert [int(v) for v in out] == pins["pcg32_seed42_stream54"]
    a, b = pins["mix64"]
    assert oracle_lib.lib().orc_mix64(a) == b


def test_sobol_first_points(oracle_lib, pins):
    for i, point in enumerate(pins["sobol_first_points_gray_order"]):
        index = i ^ (i >> 1)
        for dim, want in enumerate(point):
            assert oracle_lib.lib().orc_sobol(dim, index) / 4294967296.0 == want


def test_energy_tables_match_the_reference(oracle_lib, pins):
    t = oracle_lib.energy_tables()
    names = {"ALBEDO": "albedo", "SCHLICK": "schlick", "CLEAR_IN": "clear_in", "CLEAR_OUT": "clear_out",
             "ALBEDO_AVG": "albedo_avg", "SCHLICK_AVG": "schlick_avg"}
    for ref_name, key in names.items():
        v = t[key]
        raw = v.astype("<u2").tobytes() if v.dtype == np.uint16 else v.astype("<f4").tobytes()
        assert len(v) == pins["energy_tables"][ref_name]["count"]
        assert hashlib.sha256(raw).hexdigest() == pins["energy_tables"][ref_name]["sha256"], ref_name


def test_example_scene_bytes_are_the_reference_fixture(example_rsb, pins):
    assert len(example_rsb) == pins["example_rsb"]["bytes"]
    assert hashlib.sha256(example_rsb).hexdigest() == pins["example_rsb"]["sha256"]


def test_example_tiles_have_the_pinned_hashes(oracle_lib, example_rsb, pins):
    s = oracle_lib.OracleScene(example_rsb)
    for (x, y), key in [((240, 176), "tile_centre_240_176_s3"), ((48, 144), "tile_small_sphere_48_144_s3")]:
        out = s.render_tile(x, y, 32, 32, 3)
        assert oracle_lib.fnv1a(out) == pins["film_hashes"][key]


def test_whole_example_at_four_samples_has_the_pinned_hash(oracle_lib, example_rsb, pins):
    s = oracle_lib.OracleScene(example_rsb)
    rgb, w, _, _, _ = s.render_film(0, 4, tile=32, threads=4)
    assert oracle_lib.fnv1a(oracle_lib.resolve(rgb, w)) == pins["film_hashes"]["example_4spp"]


def pass_hashes(fnv1a, normal, depth, part, material, albedo_sum, alpha_sum, samples):
    """FNV-1a of each plane as the reference hashes them (passes.rs:529, Plane::fnv1a over the
    little-endian words): the albedo and alpha sums scaled by the f32 reciprocal of the count."""
    inv = np.float32(1.0) / np.float32(samples)
    return {
        "albedo": fnv1a((albedo_sum * inv).astype(np.float32)),
        "normal": fnv1a(normal),
        "depth": fnv1a(depth),
        "part_id": fnv1a(np.ascontiguousarray(part, np.uint32).view(np.float32)),
        "material_id": fnv1a(np.ascontiguousarray(material, np.uint32).view(np.float32)),
        "alpha": fnv1a((alpha_sum * inv).astype(np.float32)),
    }


@pytest.mark.parametrize("name", ["example", "e5_hdri"])
def test_passes_of_the_example_and_e5_have_the_pinned_hashes(oracle_lib, pins, name):
    """render/passes_tests.rs:155-194, 197-230, 840-862: the exact passes and 4 samples of albedo and
    alpha, added in sample order, of the example (512 x 384) and the E5 example with its HDRI."""
    from repackshot_b200 import scenes
    desc = scenes.example_scene() if name == "example" else scenes.e5_scene()
    o = oracle_lib.OracleScene(scenes.to_rsb(desc))
    normal, depth, part, material = o.passes()
    albedo, alpha = np.zeros_like(o.albedo(0)), np.zeros_like(o.alpha(0))
    for s in range(4):
        albedo = (albedo + o.albedo(s)).astype(np.float32)
        alpha = (alpha + o.alpha(s)).astype(np.float32)
    got = pass_hashes(oracle_lib.fnv1a, normal, depth, part, material, albedo, alpha, 4)
    want = {k: v for k, v in pins["passes_4spp"][name].items() if k != "coc"}
    assert got == want
