"""Suns, point lights, sphere lights and spots on the GPU, through the C ABI, against the oracle.

* The reference's sun-triangle known answer (render.rs:797-827): the centre pixel is 0.8 within
  1e-5, everything outside pixels 5..10 is exactly 0, and the film has the oracle's bits.
* Each kind alone and all together in the example scene: per-path radiance equals the oracle's
  (relative 1e-4; the path is built to be bit-exact and the test reports exactness), and the
  film of several samples has the oracle's bits.
* The adjoint's power gradients of a sun, a sphere light and a spot match central finite
  differences of the loss (depth 2, 4096 spp, the correlated estimate), within 1e-2.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PATH_RTOL = 1.0e-4


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def test_triangle_facing_the_sun(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.sun_triangle_scene())
    f = rtg.Scene(rsb).film()
    f.render(0, 1)
    px = f.resolve().reshape(16, 16, 3)
    assert np.all(np.abs(px[8, 8] - 0.8) < 1.0e-5), px[8, 8]
    outside = np.ones((16, 16), bool)
    outside[5:11, 5:11] = False
    assert np.all(px[outside] == 0.0)
    assert int(np.sum(px[5:11, 5:11, 0] > 0.0)) >= 8
    rgb, wt, _, _, _ = oracle_lib.OracleScene(rsb).render_film(0, 1)
    assert np.array_equal(px.view(np.uint32), oracle_lib.resolve(rgb, wt).reshape(16, 16, 3).view(np.uint32))


def variant(name):
    """The light-kinds scene (96 x 72) keeping some of its lights: 0 rect, 1 sun disc, 2 point,
    3 sphere, 4 spot; `delta sun` turns the sun into a delta direction, `dark` turns off the dome."""
    from repackshot_b200 import scenes
    s = scenes.light_kinds_scene(96, 72)
    keep = {"all": [0, 1, 2, 3, 4], "sun disc": [1], "delta sun": [1], "point": [2], "sphere": [3], "spot": [4],
            "point dark": [2], "spot and sphere dark": [3, 4], "suns and spheres": [1, 1, 3, 4, 4]}[name]
    lights = [copy.deepcopy(s.lights[i]) for i in keep]
    if name == "delta sun":
        lights[0].angle_deg = 0.0
    if name == "suns and spheres":
        lights[1].direction, lights[1].angle_deg = (0.6, -0.2, -0.77), 10.0
        lights[4].position, lights[4].direction = (400.0, -300.0, 500.0), (-0.4, 0.3, -0.87)
    s.lights = lights
    if "dark" in name:
        s.env_strength = 0.0
    return scenes.to_rsb(s)


NAMES = ["all", "sun disc", "delta sun", "point", "sphere", "spot", "point dark", "spot and sphere dark", "suns and spheres"]


@pytest.mark.parametrize("name", NAMES)
def test_paths_match_the_oracle(rtg, oracle_lib, name):
    rsb = variant(name)
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    rng = np.random.default_rng(5)
    n = 4000
    xys = np.stack([rng.integers(0, g.width, n), rng.integers(0, g.height, n), rng.integers(0, 64, n)], 1).astype(np.uint32)
    got, want = g.render_paths(xys), o.paths(xys)
    assert np.allclose(got[:, :4], want[:, :4], rtol=PATH_RTOL, atol=1e-6)
    exact = np.mean(np.all(got[:, :4].view(np.uint32) == want[:, :4].view(np.uint32), axis=1))
    print(f"{name}: {exact * 100:.2f}% of paths bit-exact")
    assert float(np.abs(want[:, :3]).sum()) > 0.0


@pytest.mark.parametrize("name", ["all", "suns and spheres"])
def test_film_has_the_oracle_bits(rtg, oracle_lib, name):
    rsb = variant(name)
    g, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    f = g.film()
    f.render(0, 8)
    rgb, w, al, l2, _ = o.render_film(0, 8, threads=8)
    for got, want in zip(f.read(), (rgb, w, al, l2)):
        assert np.array_equal(np.asarray(got).view(np.uint32), want.view(np.uint32))


def image(film):
    rgb, wt, _, _ = film.read()
    wt = wt.astype(np.float64)
    return np.where(wt[..., None] > 0, rgb / np.where(wt > 0, wt, 1.0)[..., None], 0.0)


def loss64(img, target):
    return float(np.mean((np.asarray(img, np.float64) - np.asarray(target, np.float64)) ** 2))


def test_power_gradients_of_suns_spheres_and_spots(rtg):
    from repackshot_b200 import scenes
    W, H, SPP = 64, 48, 4096
    base = scenes.light_kinds_scene(W, H)
    base.max_depth = 2
    tgt = copy.deepcopy(base)
    for j, k in zip(range(5), (1.1, 0.85, 1.2, 0.8, 1.15)):
        tgt.lights[j].power *= k
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(100_000, SPP)
    target = image(tf).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    nm, nl = s.adjoint_params()
    assert nl == 5
    _, grads, _ = s.adjoint(s.film(), target, 0, SPP, correlated=True)
    for j in (1, 3, 4):  # sun disc, sphere, spot
        out = []
        h = 0.02 * base.lights[j].power
        for sign in (1, -1):
            v = copy.deepcopy(base)
            v.lights[j].power += sign * h
            s.update(scenes.to_rsb(v, meshes=False))
            f = s.film()
            f.render(0, SPP)
            out.append(loss64(image(f), target))
        s.update(scenes.to_rsb(base, meshes=False))
        fd = (out[0] - out[1]) / (2 * h)
        g = float(grads[4 * nm + j])
        print(f"light {j}: adjoint {g:.6g} finite difference {fd:.6g}")
        assert abs(g - fd) <= 1e-2 * abs(fd)
