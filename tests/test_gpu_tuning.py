"""The tuning of a scene's waves (rtg_set_tuning, rtg_get_tuning) and the autotuner
(rtg_autotune). How rays and paths are ordered never changes a film's bits: the product scene's
materials and lights render the same film, bit for bit, with the ray sort off or at every grid,
with or without sorted shadow rays and material-sorted shading, in waves of any size, with the
last rounds in the tail kernel from any round on; and after the autotuner has chosen."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtg():
    import repackshot_b200 as rtg
    rtg.lib()
    return rtg


def bits(film):
    return [np.asarray(a).view(np.uint32).copy() for a in film.read()]


def test_every_tuning_gives_the_same_film(rtg, small_product_rsb):
    s = rtg.Scene(small_product_rsb)
    assert s.tuning() == {"ray_bits": 0, "shadow_sort": 0, "material_sort": 1, "capacity": 0, "l2_persist": 0, "tail_paths": 1 << 14}
    ref = None
    # A wave here holds 96 x 64 x 3 or x 5 paths: a tail limit of 2^16 takes every round from the
    # third on, 2000 and 100 later rounds, 1 almost none.
    for ray_bits, shadow, msort, cap, l2, tail in [(0, 0, 1, 0, 0, 0), (4, 1, 1, 0, 1, 0), (5, 1, 1, 0, 0, 0), (3, 0, 1, 0, 1, 0),
                                                   (2, 1, 0, 0, 0, 0), (1, 1, 1, 4096, 1, 0), (5, 0, 0, 20000, 0, 0), (4, 1, 1, 0, 0, 0),
                                                   (0, 0, 1, 0, 0, 1 << 16), (0, 0, 1, 0, 0, 2000), (0, 0, 1, 0, 0, 100),
                                                   (0, 0, 1, 0, 0, 1), (4, 1, 1, 4096, 0, 1 << 16), (0, 0, 0, 20000, 1, 5000)]:
        s.set_tuning(ray_bits=ray_bits, shadow_sort=shadow, material_sort=msort, capacity=cap, l2_persist=l2, tail_paths=tail)
        assert s.tuning() == {"ray_bits": ray_bits, "shadow_sort": shadow, "material_sort": msort,
                              "capacity": max(cap, 1024) if cap else 0, "l2_persist": l2, "tail_paths": tail}
        f = s.film()
        f.render(0, 3)
        f.render(3, 5)
        got = bits(f)
        if ref is None:
            ref = got
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (ray_bits, shadow, msort, cap, l2, tail)


def test_out_of_range_bits_are_refused(rtg, cfg0_rsb):
    L = rtg.lib()
    s = rtg.Scene(cfg0_rsb)
    v = np.array([6, 1, 1, 0], np.uint32)
    assert L.rtg_set_tuning(s.handle, rtg._ptr(v), 4) == rtg.STATUS_BAD_SCENE
    assert L.rtg_set_tuning(0, rtg._ptr(v), 4) == rtg.STATUS_BAD_HANDLE
    assert s.tuning()["ray_bits"] == 0


def test_autotuner_keeps_the_fastest_and_the_bits(rtg, small_product_rsb):
    s = rtg.Scene(small_product_rsb)
    ref = s.film()
    ref.render(0, 8)
    out = s.autotune(0, 4)
    tried = out["tried"]
    assert len(tried) >= 7
    # The chosen tuning was tried, and no candidate was more than 1% faster (a candidate must beat
    # the best so far by more than 1% to replace it).
    keys = ("ray_bits", "shadow_sort", "material_sort", "capacity", "l2_persist", "tail_paths")
    chosen = [t for t in tried if {k: t[k] for k in keys} == out["chosen"]]
    assert len(chosen) == 1
    assert chosen[0]["ms"] <= min(t["ms"] for t in tried) / 0.99 + 1e-9
    f = s.film()
    f.render(0, 8)
    for a, b in zip(bits(f), bits(ref)):
        assert np.array_equal(a, b)
