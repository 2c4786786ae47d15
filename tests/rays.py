"""Seeded ray batches for the traversal parity tests."""
import numpy as np


def random_rays(n, lo, hi, seed, t_min=1.0e-3, t_max=np.inf):
    """Incoherent rays: origins around the box [lo, hi] (grown by half its size), directions
    towards random points inside it; 8 floats per ray."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    c, e = (lo + hi) / 2, (hi - lo)
    o = c + (rng.random((n, 3)) - 0.5) * e * 2.0
    tgt = c + (rng.random((n, 3)) - 0.5) * e
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 3:6], r[:, 6], r[:, 7] = o, d, t_min, t_max
    return r


def edge_rays():
    """Axis-parallel and degenerate-direction rays (zero components, -0, huge t_min)."""
    rays = []
    for d in [(0, 0, -1), (0, 0, 1), (1, 0, 0), (0, -1, 0), (-0.0, 0.0, -1.0), (1e-30, 0, -1)]:
        for o in [(0, 0, 1000), (0, 0, 100), (-330, 120, 500), (50, 50, 100)]:
            rays.append((*o, *d, 1e-3, np.inf))
    rays.append((0, 0, 1000, 0, 0, -1, 1e6, np.inf))   # empty interval after t_min
    rays.append((0, 0, 1000, 0, 0, -1, 1e-3, 1e-3))    # tiny interval
    rays.append((0, 0, 1000, 0, 0, 0, 1e-3, np.inf))    # zero direction: not usable
    return np.array(rays, np.float32)


def surface_rays(oracle_scene, n, seed):
    """Secondary rays leaving surfaces, as the path tracer spawns them: for each nearest hit of a
    seeded incoherent batch, a random direction from the hit point itself and from the point
    backed off by 1e-3 along the incoming direction (the side a refracted or reflected ray can
    start on), both with t_min 1e-3. Near large flat quads the reference's slab test culls some
    hits whose triangle test alone would pass; these rays hold the traversal to that behaviour."""
    rays = random_rays(n, (-1500, -1500, 0), (1500, 1500, 2500), seed=seed)
    hits, _ = oracle_scene.trace(rays)
    m = hits[:, 0] != 0xFFFFFFFF
    r, t = rays[m], hits[m, 2].view(np.float32)
    p = (r[:, 0:3] + r[:, 3:6] * t[:, None]).astype(np.float32)
    rng = np.random.default_rng(seed + 1)
    d = rng.normal(size=(len(p), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((2 * len(p), 8), np.float32)
    out[0::2, 0:3] = p
    out[1::2, 0:3] = p - r[:, 3:6] * np.float32(1.0e-3)
    out[0::2, 3:6] = d
    out[1::2, 3:6] = d
    out[:, 6], out[:, 7] = 1.0e-3, np.inf
    return out
