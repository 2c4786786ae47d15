"""The adjoint's CPU reference (the oracle's orc_adjoint_reference) against central finite
differences of the oracle's own renders, where the two are the same derivative: the small scene
at depth 2 (no roulette, whose survival follows the throughput's largest channel) with its dome
turned off (one light, so the light choice does not depend on its power), the Lambert floor's
colour (its cosine sampling does not depend on it) and the light's power, with the same sample
indices on both sides, correlated (the derivative of the film's own loss). Where sampling does
depend on the parameter (the conductor's lobe choice between its GGX lobe and its energy
compensation follows its colour) the detached estimate and a same-seed finite difference agree
only in expectation, which the device tests check at many samples."""
import copy

import numpy as np

from repackshot_b200 import scenes

W = H = 24
SPP = 8


def scene():
    s = scenes.cfg0_scene()
    s.width, s.height, s.max_samples, s.max_depth = W, H, SPP, 2
    s.env_strength = 0.0
    return s


def loss(oracle_lib, s, target):
    rgb, wt, _, _, _ = oracle_lib.OracleScene(scenes.to_rsb(s)).render_film(0, SPP, threads=4)
    img = rgb.astype(np.float64) / wt[..., None].astype(np.float64)
    return float(np.mean((img.astype(np.float32).astype(np.float64) - target) ** 2))


def test_reference_gradient_matches_finite_differences(oracle_lib):
    base = scene()
    target = np.full((H, W, 3), 0.3, np.float32)
    o = oracle_lib.OracleScene(scenes.to_rsb(base))
    assert o.n_materials == 2 and o.n_lights == 1
    _, g = o.adjoint_reference(target, 0, SPP, threads=4, correlated=True)
    h = 1.0e-3
    checks = []
    for m in (1,):  # the floor's colour, channel by channel
        for c in range(3):
            out = []
            for sign in (1, -1):
                v = copy.deepcopy(base)
                col = list(v.materials[m].base_color)
                col[c] += sign * h
                v.materials[m].base_color = tuple(col)
                out.append(loss(oracle_lib, v, target.astype(np.float64)))
            checks.append((f"material {m} channel {c}", g[4 * m + c], (out[0] - out[1]) / (2 * h)))
    p = base.lights[0].power
    out = []
    for sign in (1, -1):
        v = copy.deepcopy(base)
        v.lights[0].power = p * (1 + sign * h)
        out.append(loss(oracle_lib, v, target.astype(np.float64)))
    checks.append(("light power", g[8], (out[0] - out[1]) / (2 * h * p)))
    for name, got, want in checks:
        assert abs(got - want) <= 2e-3 * abs(want) + 1e-9, (name, got, want)
