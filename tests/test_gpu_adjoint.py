"""The adjoint (rtg_render_adjoint) on the GPU.

- Its forward pass renders the film rtg_render_progressive renders, bit for bit, and its loss is
  the host's f64 loss of that film against the target.
- The replay retraces the forward paths: the radiance left after it is 0 up to rounding.
- Its gradients (the correlated estimate: the derivative of this very loss estimate) match
  central finite differences of the loss (same sample indices, the parameter changed through
  rtg_scene_update). The adjoint holds sampling fixed (detached sampling); a finite
  difference lets lobe choices, GGX sample directions and roulette decisions move with the
  parameter, so the two agree in expectation and differ by Monte Carlo noise that is small only
  where those decisions do not depend on the parameter. So, at depth 2 (no roulette) and 4096 spp:
  Lambert colour within 1e-2 (nothing moves: the two are equal up to rounding), conductor and glass
  colour and light power within 3e-2, GGX alpha of rough materials (alpha >= 0.3) within 8e-2; at
  the differentiable workload's depth 6, light power within 3e-2 (roulette does not depend on it).
  The alpha of sharp lobes (alpha < 0.1) has a heavy-tailed detached estimate and is not compared.
- The same check against finite differences computed on the CPU by the oracle (the reference's
  path tracer restated; loss summed in f64), on a smaller image.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, SPP, DEPTH = 64, 64, 256, 6


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def base_and_target(w=W, h=H):
    from repackshot_b200 import scenes
    return scenes.adjoint_scene(w, h, SPP, DEPTH), scenes.adjoint_scene(w, h, SPP, DEPTH, perturb_seed=3)


def image(film):
    rgb, wt, _, _ = film.read()
    wt = wt.astype(np.float64)
    return np.where(wt[..., None] > 0, rgb / np.where(wt > 0, wt, 1.0)[..., None], 0.0)


def loss64(img, target):
    return float(np.mean((np.asarray(img, np.float64) - np.asarray(target, np.float64)) ** 2))


@pytest.fixture(scope="module")
def setup(rtg):
    from repackshot_b200 import scenes
    base, tgt = base_and_target()
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(10_000, 128)
    target = image(tf).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    f = s.film()
    loss, grads, residual = s.adjoint(f, target, 0, SPP, correlated=True)
    return s, base, target, loss, grads, residual, image(f)


def test_forward_film_and_loss(rtg, setup):
    s, base, target, loss, grads, residual, img = setup
    f2 = s.film()
    f2.render(0, SPP)
    assert np.array_equal(image(f2), img)
    assert loss == pytest.approx(loss64(img, target), rel=1e-5)
    nm, nl = s.adjoint_params()
    assert (nm, nl) == (17, 3) and grads.shape == (4 * nm + nl,)
    assert np.all(np.isfinite(grads))


def test_replay_retraces_the_forward_paths(setup):
    residual = setup[5]
    assert residual[1] > 0
    assert residual[0] <= 1e-5 * residual[1]


def set_param(scene, kind, index, value):
    if kind == "power":
        scene.lights[index].power = value
    else:
        m, c = index
        if kind == "albedo":
            col = list(scene.materials[m].base_color)
            col[c] = value
            scene.materials[m].base_color = tuple(col)
        else:  # alpha
            scene.materials[m].roughness = float(np.sqrt(value))


def get_param(scene, kind, index):
    if kind == "power":
        return scene.lights[index].power
    m, c = index
    return scene.materials[m].base_color[c] if kind == "albedo" else scene.materials[m].roughness ** 2


def fd_gpu(rtg, s, base, target, kind, index, h):
    from repackshot_b200 import scenes
    out = []
    for sign in (1, -1):
        v = copy.deepcopy(base)
        set_param(v, kind, index, get_param(base, kind, index) + sign * h)
        s.update(scenes.to_rsb(v, meshes=False))
        f = s.film()
        f.render(0, SPP)
        out.append(loss64(image(f), target))
    s.update(scenes.to_rsb(base, meshes=False))
    return (out[0] - out[1]) / (2 * h)


def pick(grads, materials, column, nm=17):
    """(material, column) of the largest |gradient| among `materials`; column 3 is alpha."""
    G = grads[:4 * nm].reshape(nm, 4)
    cols = range(3) if column is None else [column]
    best = max(((m, c) for m in materials for c in cols), key=lambda mc: abs(G[mc[0], mc[1]]))
    return best, float(G[best[0], best[1]])


@pytest.fixture(scope="module")
def deep_setup(rtg):
    """Depth 2, 4096 spp: the comparisons where finite differences are a sharp reference."""
    from repackshot_b200 import scenes
    base = scenes.adjoint_scene(W, H, 4096, 2)
    tgt = scenes.adjoint_scene(W, H, 4096, 2, perturb_seed=3)
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(100_000, 4096)
    target = image(tf).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    _, grads, _ = s.adjoint(s.film(), target, 0, 4096, correlated=True)
    return s, base, target, grads


def fd_at(rtg, s, base, target, kind, index, h, spp):
    from repackshot_b200 import scenes
    out = []
    for sign in (1, -1):
        v = copy.deepcopy(base)
        set_param(v, kind, index, get_param(base, kind, index) + sign * h)
        s.update(scenes.to_rsb(v, meshes=False))
        f = s.film()
        f.render(0, spp)
        out.append(loss64(image(f), target))
    s.update(scenes.to_rsb(base, meshes=False))
    return (out[0] - out[1]) / (2 * h)


LAMBERT, GLASS, CONDUCTOR = range(10, 16), range(6, 10), range(0, 6)


@pytest.mark.parametrize("name, materials, column, rel", [
    ("lambert colour", LAMBERT, None, 1e-2),
    ("conductor colour", CONDUCTOR, None, 3e-2),
    ("glass colour", GLASS, None, 3e-2),
    ("rough alpha", "rough", 3, 8e-2),
])
def test_material_gradients_match_finite_differences(rtg, deep_setup, name, materials, column, rel):
    s, base, target, grads = deep_setup
    if materials == "rough":
        materials = [m for m in range(16) if base.materials[m].roughness ** 2 >= 0.3 and base.materials[m].ior != 1.0]
    (m, c), g = pick(grads, materials, column)
    kind = "alpha" if c == 3 else "albedo"
    fd = fd_at(rtg, s, base, target, kind, (m, c if c < 3 else 0), 0.02, 4096)
    print(f"{name} material {m} column {c}: adjoint {g:.6g} finite difference {fd:.6g}")
    assert abs(g - fd) <= rel * abs(fd)


def test_light_power_gradients_match_finite_differences(rtg, deep_setup, setup):
    s, base, target, grads = deep_setup
    for j in range(3):
        g = grads[4 * 17 + j]
        fd = fd_at(rtg, s, base, target, "power", j, 0.02 * base.lights[j].power, 4096)
        print(f"depth 2 light {j}: adjoint {g:.6g} finite difference {fd:.6g}")
        assert abs(g - fd) <= 3e-2 * abs(fd)
    # the differentiable workload's depth (6), with roulette
    s6, base6, target6, _, grads6, _, _ = setup
    for j in range(3):
        g = grads6[4 * 17 + j]
        fd = fd_at(rtg, s6, base6, target6, "power", j, 0.02 * base6.lights[j].power, SPP)
        print(f"depth 6 light {j}: adjoint {g:.6g} finite difference {fd:.6g}")
        assert abs(g - fd) <= 3e-2 * abs(fd) + 1e-2 * np.abs(grads6[4 * 17:]).max()


def test_gradients_against_the_cpu_oracle(rtg, oracle_lib):
    from repackshot_b200 import scenes
    w, h, spp, depth = 32, 32, 64, 2
    base = scenes.adjoint_scene(w, h, spp, depth)
    tgt = scenes.adjoint_scene(w, h, spp, depth, perturb_seed=3)
    o = oracle_lib.OracleScene(scenes.to_rsb(tgt))
    rgb, wt, _, _, _ = o.render_film(500, 128, threads=8)
    target = (rgb.astype(np.float64) / wt[..., None]).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    _, grads, _ = s.adjoint(s.film(), target, 0, spp, correlated=True)

    def oracle_fd(kind, index, dh):
        losses = []
        for sign in (1, -1):
            v = copy.deepcopy(base)
            set_param(v, kind, index, get_param(base, kind, index) + sign * dh)
            rgb, wt, _, _, _ = oracle_lib.OracleScene(scenes.to_rsb(v)).render_film(0, spp, threads=8)
            losses.append(loss64(rgb.astype(np.float64) / wt[..., None], target))
        return (losses[0] - losses[1]) / (2 * dh)

    j = int(np.argmax(np.abs(grads[4 * 17:])))
    fd = oracle_fd("power", j, 0.02 * base.lights[j].power)
    print(f"light {j}: adjoint {grads[4 * 17 + j]:.6g} oracle finite difference {fd:.6g}")
    assert abs(grads[4 * 17 + j] - fd) <= 3e-2 * abs(fd)
    (m, c), g = pick(grads, LAMBERT, None)
    fd = oracle_fd("albedo", (m, c), 0.02)
    print(f"lambert material {m} channel {c}: adjoint {g:.6g} oracle finite difference {fd:.6g}")
    assert abs(g - fd) <= 1e-2 * abs(fd)


def test_decorrelated_gradient_agrees_with_the_correlated_one_at_high_spp(rtg, deep_setup):
    # Both estimate the same gradient; at 4096 spp their difference (the noise covariance) is small.
    s, base, target, grads = deep_setup
    _, dec, _ = s.adjoint(s.film(), target, 0, 4096)
    big = np.abs(grads) > 0.2 * np.abs(grads).max()
    assert big.sum() >= 3
    assert np.allclose(dec[big], grads[big], rtol=0.05)
