"""rtg_scene_update (rt_scene_update, engine/crates/rt-wasm/src/ffi.rs:68-88) on the GPU: an
updated scene renders exactly what a fresh load of the same full scene renders, whether the update
keeps the device trees (camera, lights, materials, image size), rebuilds them over the kept meshes
(new instance transforms) or replaces the geometry (a file with MESH sections); a bad file leaves
the scene as it was.
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


def film_bits(scene, first=0, count=2):
    f = scene.film()
    f.render(first, count)
    return [a.copy() for a in f.read()]


def same(a, b):
    return all(np.array_equal(x.view(np.uint32), y.view(np.uint32)) for x, y in zip(a, b))


def check_update(rtg, base, changed):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(base))
    nodes, built = s.nodes, s.build_seconds
    s.update(scenes.to_rsb(changed, meshes=False))
    s.kept_trees = s.build_seconds == built
    fresh = rtg.Scene(scenes.to_rsb(changed))
    assert (s.width, s.height) == (fresh.width, fresh.height)
    assert same(film_bits(s), film_bits(fresh))
    return s, fresh, nodes


def test_camera_lights_materials_and_size_keep_the_trees(rtg):
    from repackshot_b200 import scenes
    base = scenes.example_scene()
    changed = copy.deepcopy(base)
    changed.camera_position = tuple(v * 1.1 for v in base.camera_position)
    changed.lights[0].power *= 2.5
    changed.materials[0].base_color = (0.2, 0.7, 0.3)
    changed.width, changed.height = 320, 200
    s, fresh, nodes = check_update(rtg, base, changed)
    assert s.nodes == nodes == fresh.nodes
    assert s.kept_trees  # the device trees were not built again


def test_new_instance_transforms_rebuild_over_the_kept_meshes(rtg):
    from repackshot_b200 import scenes
    base = scenes.example_scene()
    changed = copy.deepcopy(base)
    rows = list(changed.instances[0].rows)
    rows[3] += 150.0  # move the first instance along x
    changed.instances[0].rows = tuple(rows)
    check_update(rtg, base, changed)


def test_a_file_with_meshes_replaces_the_geometry(rtg, pins):
    from repackshot_b200 import scenes
    s = rtg.Scene(scenes.to_rsb(scenes.cfg0_scene()))
    s.update(scenes.to_rsb(scenes.example_scene()))
    f = s.film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["example_4spp"]


def test_a_bad_file_leaves_the_scene_unchanged(rtg, example_rsb, pins):
    s = rtg.Scene(example_rsb)
    with pytest.raises(rtg.RtgError) as e:
        s.update(b"RSB1garbage")
    assert e.value.status == rtg.STATUS_BAD_SCENE
    with pytest.raises(rtg.RtgError):
        s.update(example_rsb[:-7])
    f = s.film()
    f.render(0, 4)
    assert rtg.fnv1a(f.resolve()) == pins["film_hashes"]["example_4spp"]
