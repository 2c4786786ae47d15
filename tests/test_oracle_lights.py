"""The oracle's suns, point lights and spots against the reference's own known answers: the unit
tests of engine/crates/rt-core/src/light.rs (suns_give_their_irradiance_and_cover_their_disc,
a_point_light_gives_its_intensity_over_the_distance_squared,
a_sphere_light_lights_like_its_point_and_shows_its_radiance,
a_spot_lights_its_cone_and_fades_at_its_edge, a_narrow_spot_aimed_at_the_scene_is_chosen_like_its_point_light,
a_light_without_shadow_says_so) and render.rs:797-827
(a_triangle_facing_the_camera_lights_exactly_its_projection), restated with the same scenes,
sample points and tolerances, through the oracle's light helpers and renderer.
"""
import math

import numpy as np
import pytest

from repackshot_b200 import scenes
from repackshot_b200.scenes import LIGHT_POINT, LIGHT_SPOT, LIGHT_SUN, Light


def lights_only(*lights, env_strength=0.0, meshes=()):
    """Scene::default() with only these lights (and meshes): an empty scene's bounds are the
    sphere of radius 1000 about the origin; black_env() is the default dome at strength 0."""
    s = scenes.Scene(lights=list(lights), env_strength=env_strength, width=16, height=16)
    if meshes:
        s.materials = [scenes.Material()]
        s.meshes = list(meshes)
        s.instances = [scenes.Instance(i) for i in range(len(meshes))]
    return s


def load(oracle_lib, s):
    return oracle_lib.OracleScene(scenes.to_rsb(s))


def point(position, diameter, power):
    """light.rs:1751: a point light of that diameter, glossy, facing down."""
    return Light(kind=LIGHT_POINT, position=position, direction=(0.0, 0.0, -1.0), size_x=diameter, size_y=diameter,
                 power=power, angle_deg=0.5, flags=1)


def irradiance_up(o, x, n=64):
    """light.rs:1764: irradiance at x on a surface facing +Z by n x n stratified light samples."""
    e = 0.0
    for i in range(n):
        for j in range(n):
            s = o.light_sample(x, 0.5, ((i + 0.5) / n, (j + 0.5) / n))
            if s is not None:
                wi, _, rad, pdf, _, _ = s
                e += float(np.float32(rad[1] * max(wi[2], 0.0) / pdf))
    return e / (n * n)


def test_sun_gives_its_irradiance_and_covers_its_disc(oracle_lib):
    sun = Light(kind=LIGHT_SUN, position=(0.0, 0.0, 1000.0), direction=(0.0, 0.0, -1.0), size_x=500.0, size_y=500.0,
                power=3.0, angle_deg=0.53, flags=3)
    o = load(oracle_lib, lights_only(sun))
    e = 0.0
    for i in range(64):
        for j in range(64):
            s = o.light_sample((0.0, 0.0, 0.0), 0.3, ((i + 0.5) / 64, (j + 0.5) / 64))
            assert s is not None
            wi, dist, rad, pdf, delta, _ = s
            assert not delta and math.isinf(dist)
            assert o.light_sky(wi)[1] > 1.0e3  # inside the disc the camera sees
            e += float(np.float32(rad[1] * wi[2] / pdf))
    assert abs(e / 4096.0 - 3.0) < 1.0e-3
    assert o.light_sky((0.0, 0.0, 1.0))[1] > 1.0e3
    d = np.array([0.0, 0.1, 1.0], np.float32)
    assert np.array_equal(o.light_sky(d / np.linalg.norm(d)), np.zeros(3, np.float32))
    # A delta sun: the irradiance itself, the selection probability as its density; never seen.
    sun.angle_deg = 0.0
    o = load(oracle_lib, lights_only(sun))
    wi, dist, rad, pdf, delta, _ = o.light_sample((0.0, 0.0, 0.0), 0.9, (0.1, 0.2))
    assert delta and pdf == 1.0 and rad[1] == 3.0
    assert np.array_equal(o.light_sky((0.0, 0.0, 1.0)), np.zeros(3, np.float32))


def test_point_light_gives_its_intensity_over_the_distance_squared(oracle_lib):
    o = load(oracle_lib, lights_only(point((0.0, 0.0, 400.0), 0.0, 12.0)))
    assert o.light_count() == 1
    wi, dist, rad, pdf, delta, shadow = o.light_sample((0.0, 0.0, 0.0), 0.5, (0.3, 0.7))
    want = 12.0 / (4.0 * math.pi * 0.16)
    assert delta and pdf == 1.0 and shadow
    assert abs(rad[1] - want) < want * 1.0e-5
    assert abs(dist - 400.0) < 1.0e-3
    e = irradiance_up(o, (300.0, 0.0, 0.0))
    want = 12.0 / (4.0 * math.pi * 0.25) * 0.8
    assert abs(e / want - 1.0) < 1.0e-4
    # A point is never seen.
    assert np.array_equal(o.light_crossed((0.0, 0.0, 0.0), (0.0, 0.0, 1.0)), np.zeros(3, np.float32))


def test_sphere_light_lights_like_its_point_and_shows_its_radiance(oracle_lib):
    sphere = point((0.0, 0.0, 400.0), 100.0, 12.0)
    sphere.flags = 3
    o = load(oracle_lib, lights_only(sphere))
    e = irradiance_up(o, (0.0, 0.0, 0.0))
    want = 12.0 / (4.0 * math.pi * 0.16)
    assert abs(e / want - 1.0) < 2.0e-3
    _, dist, _, _, delta, _ = o.light_sample((0.0, 0.0, 0.0), 0.5, (0.5, 0.5))
    assert not delta and 340.0 < dist < 400.0
    radiance = 12.0 / (4.0 * math.pi) / (math.pi * 0.05 * 0.05)
    up = ((0.0, 0.0, 0.0), (0.0, 0.0, 1.0))
    assert abs(o.light_crossed(*up)[1] - radiance) < radiance * 1.0e-4
    assert np.array_equal(o.light_crossed(*up, t_max=300.0), np.zeros(3, np.float32))
    w = o.light_crossed(*up, bsdf_pdf=1.0)[1]
    assert 0.0 < w < radiance
    # From inside the sphere nothing is sampled.
    assert o.light_sample((0.0, 0.0, 390.0), 0.5, (0.5, 0.5)) is None


def _spot(spread, angle):
    s = point((0.0, 0.0, 1000.0), 0.0, 20.0)
    s.kind, s.spread_deg, s.angle_deg = LIGHT_SPOT, spread, angle
    return s


def test_spot_lights_its_cone_and_fades_at_its_edge(oracle_lib):
    o = load(oracle_lib, lights_only(_spot(60.0, 10.0)))
    on_axis = o.light_sample((0.0, 0.0, 0.0), 0.5, (0.5, 0.5))
    want = 20.0 / (4.0 * math.pi * 1.0)
    assert abs(on_axis[2][1] - want) < want * 1.0e-5

    def at(deg):
        a = math.radians(deg)
        return (float(np.float32(1000.0 * math.sin(a) / math.cos(a))), 0.0, 0.0)

    inner = o.light_sample(at(15.0), 0.5, (0.5, 0.5))
    d2 = at(15.0)[0] ** 2 + 1.0e6
    assert abs(inner[2][1] - 20.0 / (4.0 * math.pi * d2 * 1.0e-6)) < 1.0e-4
    assert o.light_sample(at(31.0), 0.5, (0.5, 0.5)) is None
    edge = o.light_sample(at(25.0), 0.5, (0.5, 0.5))
    d2 = at(25.0)[0] ** 2 + 1.0e6
    full = 20.0 / (4.0 * math.pi * d2 * 1.0e-6)
    t = (math.cos(math.radians(25.0)) - math.cos(math.radians(30.0))) / (math.cos(math.radians(20.0)) - math.cos(math.radians(30.0)))
    smooth = t * t * (3.0 - 2.0 * t)
    assert abs(edge[2][1] - full * smooth) < full * 1.0e-4
    hard = load(oracle_lib, lights_only(_spot(60.0, 0.0)))
    assert hard.light_sample(at(29.0), 0.5, (0.5, 0.5)) is not None
    assert hard.light_sample(at(31.0), 0.5, (0.5, 0.5)) is None


def test_narrow_spot_aimed_at_the_scene_is_chosen_like_its_point_light(oracle_lib):
    quad = scenes.Mesh(np.array([(-100.0, -100.0, 0.0), (100.0, -100.0, 0.0), (100.0, 100.0, 0.0)], np.float32),
                       np.zeros((3, 3), np.float32), np.array([0, 1, 2], np.uint32), 0)

    def pmf(light):
        return load(oracle_lib, lights_only(light, env_strength=1.0, meshes=[quad])).light_flux_pmf(0)

    at = (0.0, 0.0, 600.0)
    bare = pmf(point(at, 0.0, 5.0))

    def spot(direction):
        s = point(at, 0.0, 5.0)
        s.kind, s.spread_deg, s.angle_deg, s.direction = LIGHT_SPOT, 9.0, 2.0, direction
        return s

    aimed = pmf(spot((0.0, 0.0, -1.0)))
    away = pmf(spot((0.0, 0.0, 1.0)))
    assert 0.01 < bare < 0.99
    assert abs(aimed - bare) < 1.0e-6
    assert away < aimed * 0.1


def test_light_without_shadow_says_so(oracle_lib):
    p = point((0.0, 0.0, 400.0), 0.0, 12.0)
    p.flags = 1 | 4
    rect = Light(kind=0, position=(0.0, 0.0, 1000.0), direction=(0.0, 0.0, -1.0), size_x=100.0, size_y=100.0, power=1.0e-6,
                 angle_deg=0.5, flags=4)
    o = load(oracle_lib, lights_only(p, rect))
    assert not o.light_sample((0.0, 0.0, 0.0), 0.1, (0.5, 0.5))[5]
    assert not o.light_sample((0.0, 0.0, 0.0), 0.9999999, (0.5, 0.5))[5]


def test_triangle_facing_the_sun_lights_exactly_its_projection(oracle_lib):
    o = load(oracle_lib, scenes.sun_triangle_scene())
    rgb, wt, _, _, st = o.render_film(0, 1)
    assert st[0] >= 256
    px = rgb / wt[..., None]
    assert np.all(np.abs(px[8, 8] - 0.8) < 1.0e-5), px[8, 8]
    lit = 0
    for y in range(16):
        for x in range(16):
            if 5 <= x <= 10 and 5 <= y <= 10:
                lit += int(px[y, x, 0] > 0.0)
            else:
                assert np.array_equal(px[y, x], np.zeros(3, np.float32)), (x, y)
    assert lit >= 8


def test_ies_lights_are_refused(oracle_lib):
    s = lights_only(Light(kind=5, position=(0.0, 0.0, 400.0), power=1.0))
    with pytest.raises(ValueError, match="IES"):
        load(oracle_lib, s)


def emissive_quad_scene(power=2.0, flags=scenes.MATERIAL_FLAG_LIGHT):
    """light.rs:2032: two triangles of different size forming one 100 x 100 quad at z = 100,
    facing down (winding 0 2 1, 0 3 2), in an emissive material of white emission at power 2."""
    p = np.array([(-50.0, -50.0, 100.0), (50.0, -50.0, 100.0), (50.0, 50.0, 100.0), (-50.0, 50.0, 100.0)], np.float32)
    quad = scenes.Mesh(p, np.zeros((4, 3), np.float32), np.array([0, 2, 1, 0, 3, 2], np.uint32), 0)
    s = lights_only(meshes=[quad])
    s.materials = [scenes.Material(kind=scenes.MATERIAL_EMISSIVE, emission=(1.0, 1.0, 1.0), emission_power=power, flags=flags)]
    return s


def test_emissive_meshes_are_sampled_by_area(oracle_lib):
    # light.rs:2032 emissive_meshes_are_sampled_by_area: one mesh light; the irradiance at the
    # origin below it by 64 x 64 stratified samples (the selection spread over the CDF as well)
    # matches the square's form factor, 2 * 4 pi F(1/2, 1/2) for radiance 2, within 1%.
    o = load(oracle_lib, emissive_quad_scene())
    assert o.light_count() == 1
    e = 0.0
    for i in range(64):
        for j in range(64):
            sel = ((i * 64 + j) + 0.5) / 4096.0
            s = o.light_sample((0.0, 0.0, 0.0), sel, ((i + 0.5) / 64, (j + 0.5) / 64))
            assert s is not None
            wi, dist, rad, pdf, delta, shadow = s
            assert not delta and shadow and dist > 0.0
            e += float(np.float32(rad[1] * wi[2] / pdf))

    def f(x, y):
        return (x / math.sqrt(1 + x * x) * math.atan(y / math.sqrt(1 + x * x))
                + y / math.sqrt(1 + y * y) * math.atan(x / math.sqrt(1 + y * y))) / (2 * math.pi)

    want = 2.0 * 4.0 * math.pi * f(0.5, 0.5)
    assert abs(e / 4096.0 / want - 1.0) < 0.01


def test_emitters_without_the_light_flag_are_not_sampled(oracle_lib):
    o = load(oracle_lib, emissive_quad_scene(flags=0))
    assert o.light_count() == 0
    assert o.light_sample((0.0, 0.0, 0.0), 0.5, (0.5, 0.5)) is None
