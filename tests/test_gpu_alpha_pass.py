"""The alpha pass through the C ABI (rt_render_tile_alpha, engine/crates/rt-wasm/src/ffi.rs:379-418,
lib.rs:537), as the reference's own test of it does (rt-wasm/src/lib.rs:1142-1210,
the_alpha_pass_through_the_c_api_is_the_engines): the example at 70 x 45 in tiles of 32, the
coverage of samples 0..3 summed in f32 in sample order and scaled by the f32 reciprocal of the
count. Every sample's plane is the oracle's bit for bit (render.rs:590 render_tile_albedo_traced,
passes.rs:221 coverage_of); the image holds 0, 1 and soft edges; the bad handle, the oversized
tile, the pixels beyond the image's edge and the null pointer answer as the reference's do. E11
(edge sub-samples) gives the oracle's means over its sub-samples.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def tile_grid(w, h, size):
    for y in range(0, h, size):
        for x in range(0, w, size):
            yield x, y, min(size, w - x), min(size, h - y)


def test_the_alpha_pass_through_the_c_abi_is_the_oracles(oracle_lib):
    import repackshot_b200 as rtg
    from repackshot_b200 import scenes
    s = scenes.example_scene()
    s.width, s.height = 70, 45
    rsb = scenes.to_rsb(s)
    sc, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    samples = 3
    got = np.zeros((45, 70), np.float32)
    for x, y, w, h in tile_grid(70, 45, 32):
        acc = np.zeros(w * h, np.float32)
        for k in range(samples):
            st, one = rtg.tile_alpha(sc.handle, x, y, w, h, k)
            assert st == rtg.STATUS_OK
            assert np.array_equal(bits(one), bits(o.alpha(k, x, y, w, h)).reshape(-1))
            acc = (acc + one).astype(np.float32)
        got[y:y + h, x:x + w] = (acc * np.float32(1.0 / samples)).astype(np.float32).reshape(h, w)
    assert (got == 0).any() and (got == 1).any()
    assert ((got > 0) & (got < 1)).any(), "soft edges"
    assert rtg.tile_alpha(0, 0, 0, 4, 4, 0)[0] == rtg.STATUS_BAD_HANDLE
    assert rtg.tile_alpha(sc.handle, 0, 0, 4096, 4096, 0)[0] == rtg.STATUS_BAD_TILE
    st, edge = rtg.tile_alpha(sc.handle, 68, 0, 4, 1, 0)
    assert st == rtg.STATUS_OK and np.array_equal(edge[2:], np.zeros(2, np.float32))
    assert rtg.lib().rtg_render_tile_alpha(sc.handle, 0, 0, 4, 4, 0, None) == rtg.STATUS_NULL_POINTER


def test_edge_sub_samples_give_the_oracles_means(oracle_lib):
    import repackshot_b200 as rtg
    from repackshot_b200 import scenes
    s = scenes.e11_scene()
    s.width, s.height = 96, 64
    rsb = scenes.to_rsb(s)
    sc, o = rtg.Scene(rsb), oracle_lib.OracleScene(rsb)
    soft = False
    for k in (0, 5):
        st, a = rtg.tile_alpha(sc.handle, 0, 0, 96, 64, k)
        assert st == rtg.STATUS_OK
        want = o.alpha(k)
        assert np.array_equal(bits(a), bits(want).reshape(-1))
        soft = soft or bool(((want > 0) & (want < 1)).any())
    assert soft, "edge pixels hold means over their sub-samples"
