"""The exact passes and the 4-sample albedo and alpha through the C ABI (rtg_render_tile_passes,
rtg_render_tile_albedo, rtg_render_tile_alpha) carry the reference's pinned hashes for the example
and the E5 example with its HDRI (engine/crates/rt-core/src/render/passes_tests.rs:155-230, 840-868):
normal, depth, part and material ids, the circle of confusion, and the albedo and alpha of samples
0..3 added in sample order and scaled by the f32 reciprocal of the count. The device fills the
whole image in tiles of 32, as the reference's passes_of does."""
import numpy as np
import pytest

from test_oracle_pins import pass_hashes

pytestmark = pytest.mark.gpu


def tiles(w, h, size=32):
    for y in range(0, h, size):
        for x in range(0, w, size):
            yield x, y, min(size, w - x), min(size, h - y)


@pytest.mark.parametrize("name", ["example", "e5_hdri"])
def test_device_passes_have_the_pinned_hashes(oracle_lib, pins, name):
    import repackshot_b200 as rtg
    from repackshot_b200 import scenes
    desc = scenes.example_scene() if name == "example" else scenes.e5_scene()
    s = rtg.Scene(scenes.to_rsb(desc))
    w, h = s.width, s.height
    normal, depth = np.zeros((h, w, 3), np.float32), np.zeros((h, w), np.float32)
    part, material, coc = np.zeros((h, w), np.uint32), np.zeros((h, w), np.uint32), np.zeros((h, w), np.float32)
    albedo, alpha = np.zeros((h, w, 3), np.float32), np.zeros((h, w), np.float32)
    for x, y, tw, th in tiles(w, h):
        st, words = rtg.tile_passes(s.handle, x, y, tw, th, 0x3E)
        assert st == rtg.STATUS_OK
        n = tw * th
        normal[y:y + th, x:x + tw] = words[:3 * n].view(np.float32).reshape(th, tw, 3)
        depth[y:y + th, x:x + tw] = words[3 * n:4 * n].view(np.float32).reshape(th, tw)
        part[y:y + th, x:x + tw] = words[4 * n:5 * n].reshape(th, tw)
        material[y:y + th, x:x + tw] = words[5 * n:6 * n].reshape(th, tw)
        coc[y:y + th, x:x + tw] = words[6 * n:].view(np.float32).reshape(th, tw)
        for sample in range(4):
            st, a = rtg.tile_albedo(s.handle, x, y, tw, th, sample)
            assert st == rtg.STATUS_OK
            albedo[y:y + th, x:x + tw] = (albedo[y:y + th, x:x + tw] + a.reshape(th, tw, 3)).astype(np.float32)
            st, c = rtg.tile_alpha(s.handle, x, y, tw, th, sample)
            assert st == rtg.STATUS_OK
            alpha[y:y + th, x:x + tw] = (alpha[y:y + th, x:x + tw] + c.reshape(th, tw)).astype(np.float32)
    want = pins["passes_4spp"][name]
    got = pass_hashes(oracle_lib.fnv1a, normal, depth, part, material, albedo, alpha, 4)
    got["coc"] = oracle_lib.fnv1a(coc)
    assert got == want
