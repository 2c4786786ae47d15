"""The oracle's BVH traversal equals its brute force over every triangle (the reference's
geometry/tests.rs:207-226 strategy): on the example (instanced, one transformed instance), the
small benchmark scene and the product materials scene."""
import numpy as np
import pytest

from rays import edge_rays, random_rays


@pytest.mark.parametrize("which", ["example_rsb", "cfg0_rsb", "small_product_rsb"])
def test_bvh_equals_brute_force(oracle_lib, which, request):
    s = oracle_lib.OracleScene(request.getfixturevalue(which))
    rays = np.concatenate([random_rays(3000, (-1500, -1500, 0), (1500, 1500, 2500), seed=5), edge_rays()])
    for camera in (False, True):
        bvh, _ = s.trace(rays, camera=camera)
        brute, _ = s.trace(rays, camera=camera, brute=True)
        assert np.array_equal(bvh, brute)
    assert (bvh[:, 0] != 0xFFFFFFFF).sum() > 300
