"""Gradient-descent fitting on the adjoint (repackshot_b200.fit) on the differentiable workload
itself: 512 x 512, 32 spp, depth 6, the 16 base colours, 16 GGX alphas and 3 light powers of the
target perturbed by U(0.8, 1.2) (PCG32 seed 3), 200 Adam steps (step 0.02, decaying by 0.985 a
step), each on its own range of 32 samples. The fit recovers the parameters: the light powers to
within a tenth of their starting error, the colours and alphas to within three quarters of theirs
(a few materials cover few pixels, which the loss barely sees), and the loss above its noise floor
(the same render of the target scene itself) at least halves.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, SPP, DEPTH = 512, 512, 32, 6


def clean_loss(scene, target):
    f = scene.film()
    f.render(200_000, 256)
    rgb, wt, _, _ = f.read()
    img = rgb.astype(np.float64) / wt[..., None]
    return float(np.mean((img - target) ** 2))


def test_fit_recovers_the_parameters():
    import repackshot_b200 as rtg
    from repackshot_b200 import fit, scenes
    base = scenes.adjoint_scene(W, H, SPP, DEPTH)
    tgt = scenes.adjoint_scene(W, H, SPP, DEPTH, perturb_seed=3)
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(100_000, 512)
    rgb, wt, _, _ = tf.read()
    target = (rgb / wt[..., None]).astype(np.float32)
    floor = clean_loss(ts, target)
    s = rtg.Scene(scenes.to_rsb(base))
    before = clean_loss(s, target)
    want_p = np.array([l.power for l in tgt.lights])
    want_c = np.array([m.base_color for m in tgt.materials[:16]])
    want_a = np.array([m.roughness ** 2 for m in tgt.materials[:16]])
    F = fit.Fit(s, base, target, SPP, lr=0.02, decay=0.985)
    c0, a0, p0 = F.params()
    for _ in range(200):
        F.step()
    F._write()
    c1, a1, p1 = F.params()
    after = clean_loss(s, target)
    err = lambda x, want: (float(np.abs(x[0] - want).sum()), float(np.abs(x[1] - want).sum()))
    pe, ce, ae = err((p0, p1), want_p), err((c0, c1), want_c), err((a0, a1), want_a)
    print(f"light power error {pe[0]:.4g} -> {pe[1]:.4g}, colour {ce[0]:.4g} -> {ce[1]:.4g}, alpha {ae[0]:.4g} -> {ae[1]:.4g}; "
          f"loss above the floor {floor:.6g}: {before - floor:.6g} -> {after - floor:.6g}")
    assert pe[1] < 0.1 * pe[0]
    assert ce[1] < 0.75 * ce[0] and ae[1] < 0.75 * ae[0]
    assert after - floor < 0.5 * (before - floor)
