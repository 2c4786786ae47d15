"""The adjoint (rtg_render_adjoint) on the GPU.

- Its forward pass renders the film rtg_render_progressive renders, bit for bit, and its loss is
  the host's f64 loss of that film against the target.
- The replay retraces the forward paths: the radiance left after it is 0 up to rounding.
- Every gradient (16 + 1 materials' base colour and GGX alpha, 3 lights' power) matches the CPU
  reference of the same estimator (the oracle's orc_adjoint_reference: the reference's path
  tracer restated, each parameter's detached central difference, every sum in f64) within 1e-2
  relative, both the decorrelated gradient and the correlated one.
- Against central finite differences at h = 1e-3 (base colour and alpha +- 1e-3, a light's power
  +- 1e-3 of itself) of the loss the decorrelated gradient differentiates, mean((mean_A - target)
  (mean_B - target)) over two halves of the samples, half B drawn with the complemented seed
  (independent of A, so its expectation is the L2 loss of the converged image), at the differentiable workload's depth 6 over 8 independent ranges of 4096
  samples on 64 x 64 pixels: colour, alpha (alpha >= 0.1) and light power within 1e-2 relative
  plus three standard errors of the difference as the ranges measure it. The adjoint holds
  sampling fixed; the finite difference lets light choices, lobe choices and roulette move with
  the parameter (at h = 1e-3 a few of them flip, each by a whole contribution), so the two agree
  in expectation only, with that noise.
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


def pick(grads, materials, column, nm=17):
    """(material, column) of the largest |gradient| among `materials`; column 3 is alpha."""
    G = grads[:4 * nm].reshape(nm, 4)
    cols = range(3) if column is None else [column]
    best = max(((m, c) for m in materials for c in cols), key=lambda mc: abs(G[mc[0], mc[1]]))
    return best, float(G[best[0], best[1]])


LAMBERT, GLASS, CONDUCTOR = range(10, 16), range(6, 10), range(0, 6)


def test_gradients_match_the_cpu_fp64_reference(rtg, oracle_lib):
    from repackshot_b200 import scenes
    w, h, spp, depth = 48, 48, 16, DEPTH
    base = scenes.adjoint_scene(w, h, spp, depth)
    tgt = scenes.adjoint_scene(w, h, spp, depth, perturb_seed=3)
    o = oracle_lib.OracleScene(scenes.to_rsb(tgt))
    rgb, wt, _, _, _ = o.render_film(500, 64, threads=8)
    target = (rgb.astype(np.float64) / wt[..., None]).astype(np.float32)
    s = rtg.Scene(scenes.to_rsb(base))
    ref = oracle_lib.OracleScene(scenes.to_rsb(base))
    for correlated in (False, True):
        loss, grads, _ = s.adjoint(s.film(), target, 0, spp, correlated=correlated)
        rloss, rg = ref.adjoint_reference(target, 0, spp, threads=8, correlated=correlated)
        assert loss == pytest.approx(rloss, rel=1e-5)
        groups = (("colour", grads[:68].reshape(17, 4)[:, :3].reshape(-1), rg[:68].reshape(17, 4)[:, :3].reshape(-1)),
                  ("alpha", grads[3:68:4], rg[3:68:4]), ("light power", grads[68:], rg[68:]))
        for name, g, r in groups:
            g = np.asarray(g, np.float64)
            tol = 1e-2 * np.abs(r) + 1e-3 * np.abs(r).max()
            worst = int(np.argmax(np.abs(g - r) / tol))
            print(f"correlated={correlated} {name}: worst {g[worst]:.6g} against the reference's {r[worst]:.6g}")
            assert np.all(np.abs(g - r) <= tol)


REPS = 8  # independent sample ranges: the finite differences' noise is measured, not assumed


@pytest.fixture(scope="module")
def fd_setup(rtg):
    """The differentiable workload's scene at its depth, 64 x 64, in REPS independent ranges of 4096
    samples: per range the decorrelated gradient, and a function giving per range the central
    finite difference of the loss it differentiates."""
    from repackshot_b200 import scenes
    spp = 4096
    base = scenes.adjoint_scene(W, H, spp, DEPTH)
    tgt = scenes.adjoint_scene(W, H, spp, DEPTH, perturb_seed=3)
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(1_000_000, 1024)
    target = image(tf)
    s = rtg.Scene(scenes.to_rsb(base))
    grads = np.stack([s.adjoint(s.film(), target.astype(np.float32), r * spp, spp)[1] for r in range(REPS)]).astype(np.float64)
    half = spp // 2
    # half B as the adjoint draws it: the same scene rendered with the complemented seed
    s_b = rtg.Scene(scenes.to_rsb(with_seed(base, rtg.adjoint_seed_b(base.seed))))

    def split_loss(first):
        a, b = s.film(), s_b.film()
        a.render(first, half)
        b.render(first + half, spp - half)
        return float(np.mean((image(a) - target) * (image(b) - target)))

    def update(v):
        s.update(scenes.to_rsb(v, meshes=False))
        s_b.update(scenes.to_rsb(with_seed(v, rtg.adjoint_seed_b(v.seed)), meshes=False))

    def fd(kind, index, dh):
        out = []
        for sign in (1, -1):
            v = copy.deepcopy(base)
            set_param(v, kind, index, get_param(base, kind, index) + sign * dh)
            update(v)
            out.append(np.array([split_loss(r * spp) for r in range(REPS)]))
        update(base)
        return (out[0] - out[1]) / (2 * dh)

    return base, grads, fd


def with_seed(desc, seed):
    v = copy.deepcopy(desc)
    v.seed = seed
    return v


def agree(name, adj, fd):
    """The adjoint's mean over the ranges against the finite differences' mean: within 1e-2 relative
    plus three standard errors of their difference per range (the finite difference moves light,
    lobe and roulette choices with the parameter; the detached adjoint does not, so they agree in
    expectation, with a noise the ranges measure)."""
    d = adj - fd
    sem = float(np.std(d, ddof=1) / np.sqrt(len(d)))
    ma, mf = float(np.mean(adj)), float(np.mean(fd))
    print(f"{name}: adjoint {ma:.6g} finite difference {mf:.6g} (relative {abs(ma - mf) / abs(mf):.3%}, noise {sem / abs(mf):.3%})")
    assert abs(ma - mf) <= 1e-2 * abs(mf) + 3.0 * sem


@pytest.mark.parametrize("name, materials, column", [
    ("lambert colour", LAMBERT, None),
    ("conductor colour", CONDUCTOR, None),
    ("glass colour", GLASS, None),
    ("alpha", "rough", 3),
])
def test_material_gradients_match_finite_differences(fd_setup, name, materials, column):
    base, grads, fd = fd_setup
    if materials == "rough":
        materials = [m for m in range(16) if base.materials[m].roughness ** 2 >= 0.1 and base.materials[m].ior != 1.0]
    (m, c), _ = pick(grads.mean(axis=0), materials, column)
    kind = "alpha" if c == 3 else "albedo"
    agree(f"{name} material {m} column {c}", grads[:, 4 * m + c], fd(kind, (m, c if c < 3 else 0), 1.0e-3))


def test_alpha_gradient_matches_a_wider_finite_difference(fd_setup):
    """The alpha check at h = 1e-3 is dominated by its finite difference's noise: a step in alpha
    moves the sampled GGX directions, so a few paths change entirely. At h = 1e-2 that noise is
    ten times smaller against the step, and the central difference's own error (of order h^2 times
    the third derivative) stays far below 1e-2 of the gradient: within 1e-2 relative plus three
    standard errors, as the other checks."""
    base, grads, fd = fd_setup
    materials = [m for m in range(16) if base.materials[m].roughness ** 2 >= 0.1 and base.materials[m].ior != 1.0]
    (m, c), _ = pick(grads.mean(axis=0), materials, 3)
    agree(f"alpha material {m} at h = 1e-2", grads[:, 4 * m + 3], fd("alpha", (m, 0), 1.0e-2))


def test_light_power_gradients_match_finite_differences(fd_setup):
    base, grads, fd = fd_setup
    for j in range(3):
        agree(f"light {j}", grads[:, 4 * 17 + j], fd("power", j, 1.0e-3 * base.lights[j].power))


@pytest.fixture(scope="module")
def deep_setup(rtg):
    """Depth 2, 4096 spp: the correlated gradient (the derivative of this very estimate)."""
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


def test_decorrelated_gradient_agrees_with_the_correlated_one_at_high_spp(rtg, deep_setup):
    # Both estimate the same gradient; at 4096 spp their difference (the noise covariance) is small.
    s, base, target, grads = deep_setup
    _, dec, _ = s.adjoint(s.film(), target, 0, 4096)
    big = np.abs(grads) > 0.2 * np.abs(grads).max()
    assert big.sum() >= 3
    assert np.allclose(dec[big], grads[big], rtol=0.05)
