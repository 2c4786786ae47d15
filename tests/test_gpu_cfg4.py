"""The large stress workload (10 M triangles: 1000 rigid instances of a 10,000-triangle displaced
sphere, depth 16, all 16 materials, 8 light rigs, the adjoint on a crop) on the GPU at test sizes:

* its film has the oracle's bits (rel-MSE at most 1e-3 and at least 99 % of the pixels bit-equal,
  the bound of the other film tests);
* its 8 light-rig variants in one batched queue equal the plain renders of each rig, bit for bit;
* the adjoint over a crop of the image gives light-power gradients that match central finite
  differences at 4096 samples (the light selection follows the powers, so a few-sample estimate's
  own derivative is noisy; both converge to the gradient of the mean).
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 96, 54


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def rel_mse(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.mean((a - b) ** 2 / (b * b + 1e-2)))


def test_film_is_the_oracle_film(rtg, oracle_lib):
    from repackshot_b200 import scenes
    rsb = scenes.to_rsb(scenes.cfg4_scene(width=W, height=H, spp=2))
    s = rtg.Scene(rsb)
    assert s.triangles == 10_000_002
    f = s.film()
    f.render(0, 2)
    grgb, gw, gal, gl2 = f.read()
    rgb, w, al, l2, _ = oracle_lib.OracleScene(rsb).render_film(0, 2, threads=16)
    assert np.array_equal(gw, w)
    same = np.all(grgb.view(np.uint32) == rgb.view(np.uint32), axis=-1).mean()
    print(f"cfg4 96x54 2 spp: {same:.4f} of the pixels bit-equal, rel-MSE {rel_mse(grgb, rgb):.3g}")
    assert rel_mse(grgb / 2, rgb / 2) <= 1e-3 and same >= 0.99


def test_eight_rigs_in_one_queue_are_the_plain_renders(rtg):
    from repackshot_b200 import scenes
    base = scenes.cfg4_scene(width=64, height=36, spp=1)
    s = rtg.Scene(scenes.to_rsb(base))
    jobs = [scenes.to_rsb(scenes.cfg4_scene(width=64, height=36, spp=1, rig=scenes.light_rig(r), seed=1 + r), meshes=False)
            for r in range(8)]
    q = rtg.Queue(s)
    films = [q.add(b, 0, 2, 64, 36) for b in jobs]
    q.run()
    for r, (b, qf) in enumerate(zip(jobs, films)):
        s.update(b)
        f = s.film()
        f.render(0, 2)
        assert np.array_equal(np.asarray(qf.read()[0]).view(np.uint32), np.asarray(f.read()[0]).view(np.uint32)), r


def image(film):
    rgb, wt, _, _ = film.read()
    return np.where(wt[..., None] > 0, rgb / np.where(wt > 0, wt, 1.0)[..., None], 0.0).astype(np.float32)


def test_adjoint_on_a_crop_matches_finite_differences(rtg):
    """The decorrelated adjoint's light-power gradients on a 64 x 40 crop at depth 16 against
    central finite differences (h = 1e-3 of each power, the same sample indices) of the loss it
    differentiates, mean((mean_A - target)(mean_B - target)) over the two halves of the samples
    (half B from the complemented seed, as the adjoint draws it),
    over 8 independent ranges of 4096 samples: their means agree within 1e-2 relative plus three
    standard errors of their difference per range (the finite difference's light choices, which
    follow the powers, flip under the step; the adjoint's are held)."""
    from repackshot_b200 import scenes
    spp, reps = 4096, 8
    base = scenes.cfg4_scene(width=W, height=H, spp=spp, depth=16)
    target_scene = copy.deepcopy(base)
    for light in target_scene.lights:
        light.power *= 1.2
    crop = (16, 8, 64, 40)
    ts = rtg.Scene(scenes.to_rsb(target_scene))
    tf = ts.film(*crop)
    tf.render(1_000_000, 256)
    target = image(tf).astype(np.float64)
    s = rtg.Scene(scenes.to_rsb(base))
    seed_b = rtg.adjoint_seed_b(base.seed)  # half B as the adjoint draws it
    b_desc = copy.deepcopy(base)
    b_desc.seed = seed_b
    s_b = rtg.Scene(scenes.to_rsb(b_desc))
    nm, nl = s.adjoint_params()
    assert nl == len(base.lights) and nm == 17
    lg = []
    for r in range(reps):
        loss, grads, _ = s.adjoint(s.film(*crop), target.astype(np.float32), r * spp, spp)
        assert np.isfinite(loss) and np.all(np.isfinite(grads))
        lg.append(grads[4 * nm:].astype(np.float64))
    lg = np.array(lg)
    half = spp // 2
    for j in range(len(base.lights)):
        h = 1.0e-3 * base.lights[j].power
        out = []
        for sign in (1, -1):
            v = copy.deepcopy(base)
            v.lights[j].power += sign * h
            s.update(scenes.to_rsb(v, meshes=False))
            v.seed = seed_b
            s_b.update(scenes.to_rsb(v, meshes=False))
            per = []
            for r in range(reps):
                a, b = s.film(*crop), s_b.film(*crop)
                a.render(r * spp, half)
                b.render(r * spp + half, spp - half)
                per.append(float(np.mean((image(a).astype(np.float64) - target) * (image(b).astype(np.float64) - target))))
            out.append(np.array(per))
        fd = (out[0] - out[1]) / (2 * h)
        d = lg[:, j] - fd
        sem = float(np.std(d, ddof=1) / np.sqrt(reps))
        ma, mf = float(lg[:, j].mean()), float(fd.mean())
        print(f"cfg4 crop light {j}: adjoint {ma:.6g} finite difference {mf:.6g} (relative {abs(ma - mf) / abs(mf):.3%}, "
              f"noise {sem / abs(mf):.3%})")
        assert abs(ma - mf) <= 1e-2 * abs(mf) + 3.0 * sem
    s.update(scenes.to_rsb(base, meshes=False))


@pytest.mark.parametrize("graph", [False, True])
def test_a_queue_job_that_fills_waves_alone_runs_plain_and_keeps_its_bits(rtg, graph):
    """A queue job of at least 2^24 paths runs as the plain path's waves, with its own camera and
    lights, beside small jobs batched as before, whether the run is captured into a CUDA graph or
    not: every film equals its plain render bit for bit."""
    from repackshot_b200 import scenes
    base = scenes.cfg4_scene(width=64, height=36, spp=1)
    s = rtg.Scene(scenes.to_rsb(base))
    sizes = [(2048, 2048, 4, 3), (64, 36, 2, 5), (96, 54, 3, 6)]  # the first: 16,777,216 paths
    jobs = [(scenes.to_rsb(scenes.cfg4_scene(width=w, height=h, spp=n, rig=scenes.light_rig(r), seed=1 + r), meshes=False), w, h, n)
            for w, h, n, r in sizes]
    q = rtg.Queue(s)
    films = [q.add(b, 0, n, w, h) for b, w, h, n in jobs]
    q.run(graph=graph)
    for (b, w, h, n), qf in zip(jobs, films):
        s.update(b)
        f = s.film()
        f.render(0, n)
        for x, y in zip(qf.read(), f.read()):
            assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32)), (w, h)
