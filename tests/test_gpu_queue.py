"""The batched render queue (rtg_queue_*) on the GPU: every job's film has the bits the plain path
gives the same variant (a fresh load of the job's full scene rendered by rtg_render_progressive),
whatever the packing: one wave for all jobs, jobs split over several waves and row bands, jobs of
different depths, and the run captured into a CUDA graph. Jobs that change the geometry are
refused.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def variants():
    """Camera x light-rig x size x depth variants of the example scene, with sample ranges."""
    from repackshot_b200 import scenes
    base = scenes.example_scene()
    out = []
    for k in range(5):
        v = copy.deepcopy(base)
        v.camera_position = tuple(c * (1.0 + 0.07 * k) for c in base.camera_position)
        v.lights[0].power *= 1.0 + 0.5 * k
        v.materials[k % len(v.materials)].base_color = (0.9, 0.3 + 0.1 * k, 0.2)
        v.width, v.height = [(512, 384), (96, 64), (200, 150), (33, 17), (300, 90)][k]
        v.seed = 1 + k
        v.max_depth = [8, 12, 4, 8, 6][k]
        out.append((v, [(0, 4), (3, 2), (0, 5), (7, 9), (1, 1)][k]))
    return out


def sums(film):
    return [a.copy() for a in film.read()]


def plain(rtg, v, first, count):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(v))
    f = s.film()
    rays = f.render(first, count)
    return sums(f), rays


def bits_equal(a, b):
    return all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a, b))


@pytest.mark.parametrize("capacity, graph", [(0, False), (0, True), (20000, False)])
def test_jobs_match_the_plain_path(rtg, capacity, graph):
    from repackshot_b200 import scenes
    vs = variants()
    scene = rtg.Scene(scenes.to_rsb(vs[0][0]))
    if capacity:
        scene.set_path_capacity(capacity)  # forces several waves and row bands
    q = rtg.Queue(scene)
    films = [q.add(scenes.to_rsb(v, meshes=False), first, count, v.width, v.height) for v, (first, count) in vs]
    rays = q.run(graph=graph)
    want_rays = 0
    for f, (v, (first, count)) in zip(films, vs):
        want, r = plain(rtg, v, first, count)
        want_rays += r
        assert bits_equal(sums(f), want)
    assert rays == want_rays


def test_queue_reproduces_the_pinned_example(rtg, example_rsb, pins):
    s = rtg.Scene(example_rsb)
    q = rtg.Queue(s)
    from repackshot_b200 import scenes
    f = q.add(scenes.to_rsb(scenes.example_scene(), meshes=False), 0, 4, s.width, s.height)
    q.run()
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["example_4spp"]


def test_jobs_that_change_the_geometry_are_refused(rtg, example_rsb):
    from repackshot_b200 import scenes
    s = rtg.Scene(example_rsb)
    q = rtg.Queue(s)
    with pytest.raises(rtg.RtgError) as e:
        q.add(example_rsb, 0, 1, s.width, s.height)  # has MESH sections
    assert e.value.status == rtg.STATUS_BAD_SCENE
    moved = scenes.example_scene()
    rows = list(moved.instances[2].rows)
    rows[3] += 10.0
    moved.instances[2].rows = tuple(rows)
    with pytest.raises(rtg.RtgError):
        q.add(scenes.to_rsb(moved, meshes=False), 0, 1, s.width, s.height)
    assert q.run() == 0  # nothing was queued
