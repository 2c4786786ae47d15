"""Which meshes the section view caps (engine/crates/rt-core/src/geometry/solid.rs analyse, with the
weld of geometry/edges.rs:221-330): the product's host computation (rtg_mesh_solid, run on every
capped instance's mesh at load) and the oracle's give the same answer, and the expected one, on the
cases the rule tells apart. CPU only."""
import numpy as np
import pytest

from repackshot_b200 import scenes

OPEN, OUTWARD, INWARD = 0, 1, 2


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def box(lo=(-50, -50, -50), hi=(50, 50, 50), **kw):
    m = scenes.box_mesh(lo, hi, **kw)
    return m.positions.copy(), m.indices.copy()


def joined(*meshes):
    ps, ix, base = [], [], 0
    for p, i in meshes:
        ps.append(p)
        ix.append(i + base)
        base += len(p)
    return np.concatenate(ps), np.concatenate(ix)


def cube8():
    """The cube on its 8 corners (no weld needed)."""
    p, i = box()
    keys = [tuple(v) for v in p]
    uniq = sorted(set(keys))
    return np.array(uniq, np.float32), np.array([uniq.index(keys[k]) for k in i], np.uint32)


def moved(mesh, vertices, offset):
    p, i = mesh
    p = p.copy()
    p[vertices] += np.asarray(offset, np.float32)
    return p, i


def flipped(mesh, triangle):
    p, i = mesh
    i = i.copy()
    i[3 * triangle + 1], i[3 * triangle + 2] = i[3 * triangle + 2], i[3 * triangle + 1]
    return p, i


def corner_vertices(mesh, corner):
    p, _ = mesh
    return np.where((p == np.asarray(corner, np.float32)).all(axis=1))[0]


def chain_weld():
    """The corner (50, 50, 50) split into its three copies at 0, 0.9 and 1.8 times the weld tolerance
    (1e-5 of the 100 mm extent) along x: the first two and the last two weld, so all three do."""
    mesh = box()
    at = corner_vertices(mesh, (50, 50, 50))
    p, i = mesh
    p = p.copy()
    tol = np.float32(100.0) * np.float32(1.0e-5)
    p[at[1], 0] += np.float32(0.9) * tol
    p[at[2], 0] += np.float32(1.8) * tol
    return p, i


def icosphere(reverse=False):
    m = scenes.icosphere((0.0, 0.0, 100.0), 100.0, 2)
    i = m.indices.reshape(-1, 3)
    if reverse:
        i = i[:, [0, 2, 1]]
    return m.positions, i.reshape(-1)


def knot():
    positions, _, triangles = scenes.torus_knot(seg_u=64, seg_v=16)
    return positions, triangles.reshape(-1)


CASES = {
    "cube of 24 vertices, welded": (box(), OUTWARD),
    "cube of 8 vertices": (cube8(), OUTWARD),
    "cube wound inward": (box(inward=True), INWARD),
    "open box": (box(skip_faces=((2, 1),)), OPEN),
    "one triangle flipped": (flipped(box(), 5), OPEN),
    "two cubes sharing an edge": (joined(box((0, 0, 0), (100, 100, 100)), box((100, 100, 0), (200, 200, 100))), OPEN),
    "two separate cubes": (joined(box(), box((100, 100, 100), (150, 150, 150))), OUTWARD),
    "a corner moved within the tolerance": (moved(box(), corner_vertices(box(), (50, 50, 50))[:1], (3e-4, 0, 0)), OUTWARD),
    "a corner moved beyond the tolerance": (moved(box(), corner_vertices(box(), (50, 50, 50))[:1], (3e-3, 0, 0)), OPEN),
    "a corner welded through a chain": (chain_weld(), OUTWARD),
    "degenerate triangles beside a cube": (
        (box()[0], np.concatenate([box()[1], np.array([0, 0, 1, 2, 2, 2], np.uint32)])), OUTWARD),
    "a pillow of no volume": ((np.array([(0, 0, 0), (100, 0, 0), (100, 100, 0), (0, 100, 0)], np.float32),
                               np.array([0, 1, 2, 0, 2, 3, 0, 2, 1, 0, 3, 2], np.uint32)), OPEN),
    "empty": ((np.zeros((0, 3), np.float32), np.zeros(0, np.uint32)), OPEN),
    "icosphere": (icosphere(), OUTWARD),
    "icosphere wound inward": (icosphere(reverse=True), INWARD),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_the_product_and_the_oracle_tell_solids_alike(rtg, oracle_lib, name):
    (positions, indices), want = CASES[name]
    assert oracle_lib.mesh_solid(positions, indices) == want
    assert rtg.mesh_solid(positions, indices) == want


def test_a_torus_knot_and_random_soups_agree(rtg, oracle_lib):
    # A closed tube whose grid wraps around (no seam to weld); scenes.torus_knot winds its triangles
    # clockwise seen from outside, so it is inward, and outward with every triangle reversed.
    p, i = knot()
    assert rtg.mesh_solid(p, i) == oracle_lib.mesh_solid(p, i) == INWARD
    r = i.reshape(-1, 3)[:, [0, 2, 1]].reshape(-1)
    assert rtg.mesh_solid(p, r) == oracle_lib.mesh_solid(p, r) == OUTWARD
    rng = np.random.default_rng(9)
    for k in range(40):
        n = int(rng.integers(4, 40))
        p = rng.integers(-3, 4, (n, 3)).astype(np.float32) * np.float32(10.0)
        i = rng.integers(0, n, 3 * int(rng.integers(1, 60))).astype(np.uint32)
        assert rtg.mesh_solid(p, i) == oracle_lib.mesh_solid(p, i), k


def test_bad_meshes_are_refused(rtg):
    p, i = box()
    with pytest.raises(rtg.RtgError, match="status 19"):
        rtg.mesh_solid(p, np.concatenate([i, np.array([0, 1, 99], np.uint32)]))
    with pytest.raises(rtg.RtgError, match="status 19"):
        rtg.mesh_solid(p, i[:-1])
