"""Gradient-descent fitting on the adjoint (repackshot_b200.fit): starting from the
differentiable workload's scene, 60 Adam steps towards a target rendered at parameters perturbed
by +-20% at least halve the loss above its noise floor, measured on a fixed 256-spp render (the
floor: the same render of the target scene itself).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, SPP, DEPTH = 64, 64, 16, 6


def clean_loss(rtg, scene, target):
    f = scene.film()
    f.render(200_000, 256)
    rgb, wt, _, _ = f.read()
    img = rgb.astype(np.float64) / wt[..., None]
    return float(np.mean((img - target) ** 2))


def test_fit_reduces_the_loss():
    import repackshot_b200 as rtg
    from repackshot_b200 import fit, scenes
    base = scenes.adjoint_scene(W, H, SPP, DEPTH)
    tgt = scenes.adjoint_scene(W, H, SPP, DEPTH, perturb_seed=3)
    ts = rtg.Scene(scenes.to_rsb(tgt))
    tf = ts.film()
    tf.render(100_000, 512)
    rgb, wt, _, _ = tf.read()
    target = (rgb / wt[..., None]).astype(np.float32)
    floor = clean_loss(rtg, ts, target)
    s = rtg.Scene(scenes.to_rsb(base))
    before = clean_loss(rtg, s, target)
    F = fit.Fit(s, base, target, SPP, lr=0.02)
    for _ in range(60):
        F.step()
    F._write()
    after = clean_loss(rtg, s, target)
    print(f"loss above the floor {floor:.6g}: {before - floor:.6g} -> {after - floor:.6g}")
    assert after - floor < 0.5 * (before - floor)
